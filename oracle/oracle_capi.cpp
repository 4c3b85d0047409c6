// TEST INFRASTRUCTURE -- C entry points of the CPU oracle (d3q19_oracle.hpp),
// loaded with ctypes by the tests, the smoke check and the bench's CPU
// baseline.  Not part of the engine.
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>

#include "d3q19_oracle.hpp"
#include "d3q27_oracle.hpp"
#include "gray_oracle.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {
thread_local std::string g_err;

struct Handle {
    int real64;
    oracle::D3Q19<float> *f32 = nullptr;
    oracle::D3Q19<double> *f64 = nullptr;
};
}  // namespace

// ---------------------------------------------------------------- D3Q27 levels
namespace {
struct Multi {
    int real64;
    oracle::Multi27<float> *f32 = nullptr;
    oracle::Multi27<double> *f64 = nullptr;
};
template <class Fn>
auto with(void *hp, Fn fn) {
    Multi *h = (Multi *)hp;
    return h->real64 ? fn(*h->f64) : fn(*h->f32);
}
struct GrayH {
    int real64;
    oracle::Gray<float> *f32 = nullptr;
    oracle::Gray<double> *f64 = nullptr;
};
template <class Fn>
auto gwith(void *hp, Fn fn) {
    GrayH *h = (GrayH *)hp;
    return h->real64 ? fn(*h->f64) : fn(*h->f32);
}
}  // namespace

extern "C" {

int orc_last_error(char *buf, unsigned long long len) {
    if (!buf || len == 0) return 0;
    std::snprintf(buf, (size_t)len, "%s", g_err.c_str());
    return 0;
}

int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

// real64: 0 = FP32 arithmetic (the reference's update), 1 = FP64 oracle
void *orc_create(const lbm_setup *st, const lbm_geometry *geom, int real64) {
    try {
        Handle *h = new Handle();
        h->real64 = real64;
        if (real64) { h->f64 = new oracle::D3Q19<double>(); h->f64->create(*st, geom); }
        else { h->f32 = new oracle::D3Q19<float>(); h->f32->create(*st, geom); }
        return h;
    } catch (const std::exception &e) {
        g_err = e.what();
        return nullptr;
    }
}

void orc_destroy(void *hp) {
    Handle *h = (Handle *)hp;
    if (!h) return;
    delete h->f32;
    delete h->f64;
    delete h;
}

int orc_run(void *hp, const lbm_step_in *steps, unsigned long long n, double *forces) {
    Handle *h = (Handle *)hp;
    for (unsigned long long k = 0; k < n; k++) {
        std::array<double, 6> f = h->real64 ? h->f64->step(steps[k]) : h->f32->step(steps[k]);
        if (forces) std::memcpy(forces + 6 * k, f.data(), 6 * sizeof(double));
    }
    return 0;
}

int orc_step_slab(void *hp, unsigned z0, unsigned z1) {
    Handle *h = (Handle *)hp;
    if (h->real64) h->f64->step_slab(z0, z1); else h->f32->step_slab(z0, z1);
    return 0;
}

int orc_macros(void *hp, double *out) {
    Handle *h = (Handle *)hp;
    if (h->real64) h->f64->macros(out); else h->f32->macros(out);
    return 0;
}

unsigned long long orc_nrec(void *hp) {
    Handle *h = (Handle *)hp;
    return h->real64 ? h->f64->recs.size() : h->f32->recs.size();
}

unsigned long long orc_nface(void *hp) {
    Handle *h = (Handle *)hp;
    return h->real64 ? h->f64->faces.size() : h->f32->faces.size();
}

int orc_records(void *hp, uint32_t *out) {
    Handle *h = (Handle *)hp;
    if (h->real64) h->f64->record_words(out); else h->f32->record_words(out);
    return 0;
}

int orc_flags(void *hp, uint32_t *out) {
    Handle *h = (Handle *)hp;
    const std::vector<uint32_t> &f = h->real64 ? h->f64->flags : h->f32->flags;
    std::memcpy(out, f.data(), f.size() * 4);
    return 0;
}

int orc_faces(void *hp, uint32_t *out) {
    Handle *h = (Handle *)hp;
    const std::vector<uint32_t> &f = h->real64 ? h->f64->faces : h->f32->faces;
    std::memcpy(out, f.data(), f.size() * 4);
    return 0;
}

int orc_raw(void *hp, double *out) {
    Handle *h = (Handle *)hp;
    if (h->real64) h->f64->raw(out); else h->f32->raw(out);
    return 0;
}

unsigned long long orc_steps_done(void *hp) {
    Handle *h = (Handle *)hp;
    return h->real64 ? h->f64->steps_done : h->f32->steps_done;
}

// the FP16 / BF16 conversions and the stochastic rounding, exposed so the
// tests can check them against known values
// The constant tables the oracle computes with, for the test that pins them
// against the reference's source text: D3Q19 velocities (3 ints each),
// opposites, weights and record layout {RS, R_MASK, R_CELL, R_Q, R_FPOST,
// R_MACRO, R_FT}; D3Q27 velocities, opposites, slots, weights and
// {RS, R_MASK, R_CELL, R_Q, R_FT, MW, T_FLUID, T_SOLID, T_FACE, T_GHOST,
// T_RESTRICT}; scalars {FP16_SCALE, STEP_SEED_MUL, SEED_SRC_MUL, SEED_MW_MUL}.
int orc_tables(int *c19, int *opp19, double *w19, uint32_t *rec19, int *c27, int *opp27, int *slot27, double *w27, uint32_t *rec27,
               double *scalars) {
    for (int i = 0; i < 19; i++) {
        for (int k = 0; k < 3; k++) c19[3 * i + k] = oracle::C19[i][k];
        opp19[i] = oracle::opp19(i);
        w19[i] = oracle::weight19(i);
    }
    const uint32_t r19[7] = {oracle::RS, oracle::R_MASK, oracle::R_CELL, oracle::R_Q, oracle::R_FPOST, oracle::R_MACRO, oracle::R_FT};
    for (int k = 0; k < 7; k++) rec19[k] = r19[k];
    namespace q = oracle::q27;
    for (int i = 0; i < 27; i++) {
        c27[3 * i] = q::cx(i);
        c27[3 * i + 1] = q::cy(i);
        c27[3 * i + 2] = q::cz(i);
        opp27[i] = q::opp(i);
        slot27[i] = q::slot(i);
        w27[i] = q::weight(i);
    }
    const uint32_t r27[11] = {q::RS, q::R_MASK, q::R_CELL, q::R_Q, q::R_FT, q::MW, q::T_FLUID, q::T_SOLID, q::T_FACE, q::T_GHOST, q::T_RESTRICT};
    for (int k = 0; k < 11; k++) rec27[k] = r27[k];
    scalars[0] = oracle::FP16_SCALE;
    scalars[1] = oracle::STEP_SEED_MUL;
    scalars[2] = q::SEED_SRC_MUL;
    scalars[3] = q::SEED_MW_MUL;
    return 0;
}
uint32_t orc_sr_hash(uint32_t key, uint32_t seed) { return oracle::sr_hash(key, seed); }
uint16_t orc_f32_to_f16(float x) { return oracle::f32_to_f16(x); }
float orc_f16_to_f32(uint16_t h) { return oracle::f16_to_f32(h); }
uint16_t orc_f16_bits_ref(float x) { return oracle::f16_bits_ref(x); }
uint16_t orc_f32_to_bf16(float x) { return oracle::f32_to_bf16(x); }
float orc_sround16(float x, uint32_t key, uint32_t seed) { return oracle::sround16(x, key, seed); }


void *m27_create_probes(const lbm_multi_setup *st, const lbm_geometry *geom, const lbm_probes *probes, int real64) {
    Multi *h = new Multi();
    h->real64 = real64;
    try {
        if (real64) { h->f64 = new oracle::Multi27<double>(); h->f64->create(*st, geom, probes); }
        else { h->f32 = new oracle::Multi27<float>(); h->f32->create(*st, geom, probes); }
        return h;
    } catch (const std::exception &e) {
        g_err = e.what();
        delete h->f32;
        delete h->f64;
        delete h;
        return nullptr;
    }
}
void *m27_create(const lbm_multi_setup *st, const lbm_geometry *geom, int real64) { return m27_create_probes(st, geom, nullptr, real64); }
int m27_reset_samples(void *hp) { return with(hp, [](auto &m) { m.reset_samples(); return 0; }); }
int m27_vertex_means(void *hp, float *out) { return with(hp, [&](auto &m) { m.vertex_means(out); return 0; }); }
int m27_slice_means(void *hp, float *out) { return with(hp, [&](auto &m) { m.slice_means(out); return 0; }); }
unsigned m27_nvert(void *hp) { return with(hp, [](auto &m) { return (unsigned)m.pverts.size(); }); }
unsigned m27_npix(void *hp) { return with(hp, [](auto &m) { return (unsigned)m.npix; }); }

void m27_destroy(void *hp) {
    Multi *h = (Multi *)hp;
    if (!h) return;
    delete h->f32;
    delete h->f64;
    delete h;
}

int m27_run(void *hp, const lbm_step_in *steps, unsigned long long n, double *forces) {
    try {
        return with(hp, [&](auto &m) {
            auto out = m.run(steps, (size_t)n);
            if (forces)
                for (size_t k = 0; k < out.size(); k++) std::memcpy(forces + 6 * k, out[k].data(), 6 * sizeof(double));
            return 0;
        });
    } catch (const std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

unsigned m27_levels(void *hp) { return with(hp, [](auto &m) { return (unsigned)m.levels(); }); }

int m27_dims(void *hp, uint32_t *out) {
    return with(hp, [&](auto &m) {
        for (size_t l = 0; l < m.lv.size(); l++) { out[3 * l] = m.lv[l].NX; out[3 * l + 1] = m.lv[l].NY; out[3 * l + 2] = m.lv[l].NZ; }
        return 0;
    });
}

int m27_macros(void *hp, unsigned level, float *out) {
    return with(hp, [&](auto &m) { m.macros(level, out); return 0; });
}

unsigned long long m27_nrec(void *hp) { return with(hp, [](auto &m) { return (unsigned long long)m.nrec; }); }

int m27_records(void *hp, uint32_t *out) {
    return with(hp, [&](auto &m) { std::memcpy(out, m.rec_words.data(), m.rec_words.size() * 4); return 0; });
}

int m27_flags(void *hp, unsigned level, uint32_t *out) {
    return with(hp, [&](auto &m) { std::memcpy(out, m.lv[level].flags.data(), m.lv[level].flags.size() * 4); return 0; });
}

unsigned long long m27_fine_steps(void *hp) { return with(hp, [](auto &m) { return (unsigned long long)m.fine_steps; }); }

// ---------------------------------------------------------------- gray level
void *gray_create(const lbm_gray_setup *st, int real64) {
    GrayH *h = new GrayH();
    h->real64 = real64;
    try {
        if (real64) { h->f64 = new oracle::Gray<double>(); h->f64->create(*st); }
        else { h->f32 = new oracle::Gray<float>(); h->f32->create(*st); }
        return h;
    } catch (const std::exception &e) {
        g_err = e.what();
        delete h->f32;
        delete h->f64;
        delete h;
        return nullptr;
    }
}

void gray_destroy(void *hp) {
    GrayH *h = (GrayH *)hp;
    if (!h) return;
    delete h->f32;
    delete h->f64;
    delete h;
}

int gray_set_field(void *hp, const double *gamma) { return gwith(hp, [&](auto &g) { g.set_field(gamma); return 0; }); }
int gray_reset(void *hp) { return gwith(hp, [&](auto &g) { g.reset(); return 0; }); }

int gray_run(void *hp, unsigned long long n, double *forces) {
    return gwith(hp, [&](auto &g) {
        for (unsigned long long k = 0; k < n; k++) {
            auto f = g.step();
            if (forces) std::memcpy(forces + 6 * k, f.data(), 6 * sizeof(double));
        }
        return 0;
    });
}

int gray_backward(void *hp, const lbm_adjoint_spec *sp, double *J, double *grad) {
    return gwith(hp, [&](auto &g) { *J = g.backward(*sp, grad); return 0; });
}

}  // extern "C"
