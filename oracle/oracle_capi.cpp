// TEST INFRASTRUCTURE -- C entry points of the CPU oracle (d3q19_oracle.hpp),
// loaded with ctypes by the tests, the smoke check and the bench's CPU
// baseline.  Not part of the engine.
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>

#include "d3q19_oracle.hpp"

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
uint16_t orc_f32_to_f16(float x) { return oracle::f32_to_f16(x); }
float orc_f16_to_f32(uint16_t h) { return oracle::f16_to_f32(h); }
uint16_t orc_f16_bits_ref(float x) { return oracle::f16_bits_ref(x); }
uint16_t orc_f32_to_bf16(float x) { return oracle::f32_to_bf16(x); }
float orc_sround16(float x, uint32_t key, uint32_t seed) { return oracle::sround16(x, key, seed); }

}  // extern "C"
