"""The oracle's and the engine's constant tables against the reference's
source text.

tests/golden/reference_constants.json is written by
tests/golden/make_reference_constants.py, which reads the tables out of the
reference's own files (crates/cfd/src/shader.rs:22-73 velocity set, weights,
record layout and FP16 scale; shader.rs:507-517 the stochastic-rounding hash
and noise; lattice.rs:172-189 f16_bits; lattice.rs:676 the step seed;
d3q27.rs:1-29; mshader.rs:32-48; mlattice.rs:704).  These tests compare every
table with the oracle (liboracle.so) and with the engine's headers (a host
program compiled with nvcc that calls the engine's constexpr tables and its
hash), and run the golden vectors of sround and f16_bits through the oracle.
No GPU needed.
"""
import ctypes as C
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLD = json.loads((ROOT / "tests" / "golden" / "reference_constants.json").read_text())


def oracle_tables():
    from oracle import library

    L = library()
    c19, o19, w19, r19 = (C.c_int * 57)(), (C.c_int * 19)(), (C.c_double * 19)(), (C.c_uint32 * 7)()
    c27, o27, s27, w27, r27 = (C.c_int * 81)(), (C.c_int * 27)(), (C.c_int * 27)(), (C.c_double * 27)(), (C.c_uint32 * 11)()
    sc = (C.c_double * 4)()
    assert L.orc_tables(c19, o19, w19, r19, c27, o27, s27, w27, r27, sc) == 0
    k19 = ["RS", "R_MASK", "R_CELL", "R_Q", "R_FPOST", "R_MACRO", "R_FT"]
    k27 = ["RS", "R_MASK", "R_CELL", "R_Q", "R_FT", "MW", "T_FLUID", "T_SOLID", "T_FACE", "T_GHOST", "T_RESTRICT"]
    return {
        "d3q19": {"c": np.array(c19).reshape(19, 3).tolist(), "opp": list(o19), "weight": list(w19), "record": dict(zip(k19, r19)),
                  "fp16_scale": sc[0]},
        "step_seed_mul": int(sc[1]),
        "d3q27": {"c": np.array(c27).reshape(27, 3).tolist(), "opp": list(o27), "slot": list(s27), "weight": list(w27),
                  "record": dict(zip(k27, r27)), "seed": {"src_mul": int(sc[2]), "mw_mul": int(sc[3])}},
    }


def check_tables(t):
    g19, g27 = GOLD["d3q19"], GOLD["d3q27"]
    assert t["d3q19"]["c"] == g19["c"]
    assert t["d3q19"]["opp"] == g19["opp"]
    assert np.allclose(t["d3q19"]["weight"], g19["weight"], rtol=1e-15, atol=0)
    assert t["d3q19"]["record"] == g19["record"]
    assert t["d3q19"]["fp16_scale"] == g19["fp16_scale"]
    assert t["step_seed_mul"] == GOLD["step_seed_mul"] == g27["seed"]["step_mul"]
    assert t["d3q27"]["c"] == g27["c"]
    assert t["d3q27"]["opp"] == g27["opp"]
    assert t["d3q27"]["slot"] == g27["slot"]
    assert np.allclose(t["d3q27"]["weight"], g27["weight"], rtol=1e-15, atol=0)
    assert t["d3q27"]["record"] == g27["record"]
    assert t["d3q27"]["seed"]["src_mul"] == g27["seed"]["src_mul"]
    assert t["d3q27"]["seed"]["mw_mul"] == g27["seed"]["mw_mul"]


def test_fixture_is_self_consistent():
    # the D3Q19 opposites and the D3Q27 rules as the reference states them
    c = np.array(GOLD["d3q19"]["c"])
    assert all((c[i] == -c[o]).all() for i, o in enumerate(GOLD["d3q19"]["opp"]))
    assert abs(sum(GOLD["d3q19"]["weight"]) - 1.0) < 1e-15
    c27 = np.array(GOLD["d3q27"]["c"])
    assert all((c27[i] == -c27[o]).all() for i, o in enumerate(GOLD["d3q27"]["opp"]))
    assert abs(sum(GOLD["d3q27"]["weight"]) - 1.0) < 1e-15
    assert GOLD["d3q27"]["c"][GOLD["d3q27"]["rest"]] == [0, 0, 0]


def test_oracle_tables_match_reference_source():
    check_tables(oracle_tables())


def test_oracle_sround_and_f16_bits_match_golden_vectors():
    from oracle import library

    L = library()
    L.orc_sr_hash.argtypes = [C.c_uint32, C.c_uint32]
    L.orc_sr_hash.restype = C.c_uint32
    for key, seed, h in GOLD["golden"]["sr_hash"]:
        assert L.orc_sr_hash(key, seed) == h
    for x, key, seed, want in GOLD["golden"]["sround"]:
        got = L.orc_sround16(x, key, seed)
        assert np.float32(got) == np.float32(want), (x, key, seed, got, want)
    for x, bits in GOLD["golden"]["f16_bits"]:
        assert L.orc_f16_bits_ref(x) == bits, (x, bits)


@pytest.fixture(scope="module")
def engine_tables(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not found")
    out = tmp_path_factory.mktemp("probe") / "probe"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "--expt-relaxed-constexpr", "-o", str(out),
                    str(ROOT / "tests" / "engine_tables_probe.cu")], check=True, capture_output=True)
    pairs = GOLD["golden"]["sr_hash"]
    inp = f"{len(pairs)}\n" + "".join(f"{k} {s}\n" for k, s, _ in pairs)
    r = subprocess.run([str(out)], input=inp, capture_output=True, text=True, check=True)
    return json.loads(r.stdout)


def test_engine_tables_match_reference_source(engine_tables):
    check_tables(engine_tables)


def test_engine_hash_matches_reference_source(engine_tables):
    assert engine_tables["sr_hash"] == GOLD["golden"]["sr_hash"]
