"""Writes tests/golden/reference_constants.json from the reference's source text.

The reference cannot run here (Rust on wgpu's Metal backend), so the oracle's
and the engine's constant tables are pinned to what the reference's source
says, read from the source files themselves:

* crates/cfd/src/shader.rs:22-60  the D3Q19 velocity table `C`, `opp`, `weight`
* crates/cfd/src/shader.rs:62-73  the wall-record layout and `FP16_SCALE`
* crates/cfd/src/shader.rs:507-517  `sround`: hash constants, noise scale,
  exponent floor and clamp of the FP16 stochastic rounding
* crates/cfd/src/lattice.rs:172-189  `f16_bits` (golden vectors of its rounding)
* crates/cfd/src/lattice.rs:676  the step seed multiplier
* crates/cfd/src/d3q27.rs:1-29  the D3Q27 velocity, opposite, weight and slot rules
* crates/cfd/src/mshader.rs:32-48  the D3Q27 record layout and cell types
* crates/cfd/src/mlattice.rs:704  the D3Q27 step seed terms

Each item is matched by a pattern that spells out the reference's expression;
if the source changes shape, the script stops instead of guessing.  Golden
vectors of `sround` and `f16_bits` come from a restatement of those two
functions (numpy float32 arithmetic, one operation at a time) using the
constants read here.

    python tests/golden/make_reference_constants.py [reference root]
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "reference_constants.json"


def need(pat: str, text: str, what: str, flags=re.S) -> re.Match:
    m = re.search(pat, text, flags)
    if not m:
        raise SystemExit(f"pattern for {what} not found in the reference source")
    return m


def num(tok: str) -> int:
    return int(tok.replace("_", ""), 0)


def rust_int_expr(expr: str):
    """A Rust integer expression of `i` (the d3q27.rs forms) as a Python function."""
    py = re.sub(r"\s+as\s+(i32|usize|u32)", "", expr).replace("/", "//")
    if not re.fullmatch(r"[\si0-9()+\-*%/]+", py):
        raise SystemExit(f"unexpected expression {expr!r}")
    return eval("lambda i: " + py)  # noqa: S307 -- digits, i and arithmetic only (checked above)


def parse(root: Path) -> dict:
    src = root / "crates" / "cfd" / "src"
    shader = (src / "shader.rs").read_text()
    lattice = (src / "lattice.rs").read_text()
    d27 = (src / "d3q27.rs").read_text()
    msh = (src / "mshader.rs").read_text()
    mlat = (src / "mlattice.rs").read_text()

    # ---- D3Q19
    blk = need(r"pub const C: \[\[i32; 3\]; 19\] = \[(.*?)\];", shader, "C").group(1)
    c19 = [[int(a), int(b), int(c)] for a, b, c in re.findall(r"\[(-?\d+),\s*(-?\d+),\s*(-?\d+)\]", blk)]
    assert len(c19) == 19
    need(r"pub const fn opp\(i: usize\) -> usize \{\s*if i == 0 \{\s*0\s*\} else if i % 2 == 1 \{\s*i \+ 1\s*\} else \{\s*i - 1\s*\}",
         shader, "opp")
    opp19 = [0 if i == 0 else (i + 1 if i % 2 == 1 else i - 1) for i in range(19)]
    wb = need(r"pub fn weight\(i: usize\) -> f64 \{\s*match i \{(.*?)\}\s*\}", shader, "weight").group(1)
    arms = re.findall(r"([0-9_.=]+|_)\s*=>\s*([\d.]+)\s*/\s*([\d.]+)", wb)
    assert len(arms) == 3

    def w19(i):
        for pat, a, b in arms:
            if pat == "_":
                return float(a) / float(b)
            if "..=" in pat:
                lo, hi = pat.split("..=")
                if int(lo) <= i <= int(hi):
                    return float(a) / float(b)
            elif int(pat) == i:
                return float(a) / float(b)
        raise AssertionError

    rec19 = {k: int(v) for k, v in re.findall(r"pub const (RS|R_MASK|R_CELL|R_Q|R_FPOST|R_MACRO|R_FT): u32 = (\d+);", shader)}
    assert len(rec19) == 7
    fp16_scale = float(need(r"pub const FP16_SCALE: f64 = ([\d.]+);", shader, "FP16_SCALE").group(1))

    # ---- sround (shader.rs COMMON)
    sr = need(r"fn sround\(x: f32, key: u32\) -> f32 \{(.*?)\n\}", shader, "sround").group(1)
    m = need(r"var h = \(key \* (0x[0-9A-Fa-f]+)u\) \^ \(st\.p1 \* (0x[0-9A-Fa-f]+)u \+ (0x[0-9A-Fa-f]+)u\);", sr, "sround seed mix")
    key_mul, seed_mul, seed_add = (num(g) for g in m.groups())
    m = need(r"h \^= h >> (\d+)u; h \*= (0x[0-9A-Fa-f]+)u; h \^= h >> (\d+)u; h \*= (0x[0-9A-Fa-f]+)u; h \^= h >> (\d+)u;", sr, "sround mixer")
    s1, m1, s2, m2, s3 = (num(g) for g in m.groups())
    m = need(r"let r = f32\(h >> (\d+)u\) \* \(1\.0 / (\d+)\.0\) - 0\.5;", sr, "sround noise")
    r_shift, r_den = num(m.group(1)), num(m.group(2))
    m = need(r"let ulp = exp2\(f32\(max\(e, -(\d+)\) - (\d+)\)\);", sr, "sround ulp")
    e_floor, mant_bits = -num(m.group(1)), num(m.group(2))
    m = need(r"return clamp\(x \+ r \* ulp, -(\d+)\.0, (\d+)\.0\);", sr, "sround clamp")
    clamp = float(m.group(2))
    assert float(m.group(1)) == clamp

    # ---- f16_bits (lattice.rs:172-189)
    fb = need(r"fn f16_bits\(x: f32\) -> u16 \{(.*?)\n\}", lattice, "f16_bits").group(1)
    need(r"let exp = \(\(b >> 23\) & 0xff\) as i32 - 127 \+ 15;", fb, "f16_bits exponent")
    need(r"let man = b & 0x7f_ffff;", fb, "f16_bits mantissa")
    need(r"if man & 0x1000 != 0 \{\s*h \+= 1;", fb, "f16_bits rounding")
    step_seed = num(need(r"let seed = \(self\.steps_done as u32\)\.wrapping_add\(slot\)\.wrapping_mul\(([\d_]+)\);", lattice, "step seed").group(1))

    # ---- D3Q27
    q27 = int(need(r"pub const Q: usize = (\d+);", d27, "Q").group(1))
    rest = int(need(r"pub const REST: usize = (\d+);", d27, "REST").group(1))
    m = need(r"pub const fn c\(i: usize\) -> \[i32; 3\] \{\s*\[(.*?)\]\s*\}", d27, "c")
    parts = [p.strip() for p in re.split(r",(?![^()]*\))", m.group(1))]
    cf = [rust_int_expr(p) for p in parts]
    c27 = [[f(i) for f in cf] for i in range(q27)]
    oppf = rust_int_expr(need(r"pub const fn opp\(i: usize\) -> usize \{\s*(.*?)\s*\}", d27, "opp27").group(1))
    opp27 = [oppf(i) for i in range(q27)]
    wb = need(r"match v\[0\]\.abs\(\) \+ v\[1\]\.abs\(\) \+ v\[2\]\.abs\(\) \{(.*?)\}", d27, "weight27").group(1)
    warms = {p: float(a) / float(b) for p, a, b in re.findall(r"(\d+|_)\s*=>\s*([\d.]+)\s*/\s*([\d.]+)", wb)}
    w27 = [warms.get(str(sum(abs(v) for v in c)), warms["_"]) for c in c27]
    need(r"pub const fn slot\(i: usize\) -> usize \{\s*if i < REST \{\s*i\s*\} else \{\s*i - 1\s*\}", d27, "slot")
    slot27 = [i if i < rest else i - 1 for i in range(q27)]
    rec27 = {k: int(v) for k, v in re.findall(r"pub const (RS|R_MASK|R_CELL|R_Q|R_FT|MW|T_FLUID|T_SOLID|T_FACE|T_GHOST|T_RESTRICT): u32 = (\d+);", msh)}
    assert len(rec27) == 11
    fp16_scale27 = float(need(r"pub const FP16_SCALE: f64 = ([\d.]+);", msh, "FP16_SCALE 27").group(1))
    m = need(r"seed: \(self\.fine_steps as u32\)\.wrapping_add\(hslot\)\.wrapping_mul\(([\d_]+)\)\.wrapping_add\(src \* (\d+) \+ mw \* (\d+)\)",
             mlat, "multi-level seed")
    seed27 = [num(g) for g in m.groups()]

    consts = {
        "d3q19": {"c": c19, "opp": opp19, "weight": [w19(i) for i in range(19)], "record": rec19, "fp16_scale": fp16_scale},
        "sround": {"key_mul": key_mul, "seed_mul": seed_mul, "seed_add": seed_add, "shifts": [s1, s2, s3], "muls": [m1, m2],
                   "noise_shift": r_shift, "noise_den": r_den, "exp_floor": e_floor, "mant_bits": mant_bits, "clamp": clamp},
        "step_seed_mul": step_seed,
        "d3q27": {"q": q27, "rest": rest, "c": c27, "opp": opp27, "weight": w27, "slot": slot27, "record": rec27,
                  "fp16_scale": fp16_scale27, "seed": {"step_mul": seed27[0], "src_mul": seed27[1], "mw_mul": seed27[2]}},
    }
    consts["golden"] = golden(consts)
    return consts


# ---------------------------------------------------------------- golden vectors
M32 = 0xFFFFFFFF


def sr_hash(key: int, seed: int, k: dict) -> int:
    h = ((key * k["key_mul"]) & M32) ^ ((seed * k["seed_mul"] + k["seed_add"]) & M32)
    s1, s2, s3 = k["shifts"]
    m1, m2 = k["muls"]
    h ^= h >> s1
    h = (h * m1) & M32
    h ^= h >> s2
    h = (h * m2) & M32
    h ^= h >> s3
    return h


def sround(x: float, key: int, seed: int, k: dict) -> float:
    f = np.float32
    h = sr_hash(key, seed, k)
    r = f(h >> k["noise_shift"]) * (f(1.0) / f(k["noise_den"])) - f(0.5)
    bits = int(np.array([x], dtype=np.float32).view(np.uint32)[0])
    e = ((bits >> 23) & 0xFF) - 127
    ulp = f(np.ldexp(1.0, max(e, k["exp_floor"]) - k["mant_bits"]))
    v = f(x) + f(r * ulp)
    return float(min(max(v, f(-k["clamp"])), f(k["clamp"])))


def f16_bits(x: float) -> int:
    b = int(np.array([x], dtype=np.float32).view(np.uint32)[0])
    sign = (b >> 16) & 0x8000
    exp = ((b >> 23) & 0xFF) - 127 + 15
    man = b & 0x7FFFFF
    if exp <= 0:
        return sign
    if exp >= 31:
        return sign | 0x7C00
    h = sign | (exp << 10) | (man >> 13)
    if man & 0x1000:
        h += 1
    return h & 0xFFFF


def golden(c: dict) -> dict:
    rng = np.random.default_rng(20260101)
    keys = [int(v) for v in rng.integers(0, 2**32, 24, dtype=np.uint64)] + [0, 1, 19, 2**32 - 1]
    seeds = [int(v) for v in rng.integers(0, 2**32, 24, dtype=np.uint64)] + [0, c["step_seed_mul"], 7, 2**31]
    k = c["sround"]
    xs = [float(np.float32(v)) for v in np.concatenate([rng.normal(0, 30, 20), rng.normal(0, 3e3, 6), [0.0, 1.5e-4, -6.1e-5, 64999.0, -70000.0, 3.0]])]
    hashes = [[a, b, sr_hash(a, b, k)] for a, b in zip(keys, seeds)]
    srounds = [[x, a, b, sround(x, a, b, k)] for x, a, b in zip(xs, keys + keys, seeds + seeds)]
    fvals = [float(np.float32(v)) for v in np.concatenate([rng.normal(0, 1, 20), [0.5, 1.0, 1e-3, 0.999, 1.0009765625, 6.2e-5, 7e4, -2.5]])]
    f16 = [[x, f16_bits(x)] for x in fvals]
    return {"sr_hash": hashes, "sround": srounds, "f16_bits": f16}


def main() -> None:
    root = Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference")
    consts = parse(root)
    OUT.write_text(json.dumps(consts, indent=1) + "\n")
    print(OUT)


if __name__ == "__main__":
    main()
