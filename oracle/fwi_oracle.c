/*
 * fwi_oracle.c — CPU oracle of the FWI2D wave-propagation path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (fwi2d_b200/, the
 * executables, libfwi2d.so) may include, link or call this file; only the
 * tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, and
 * only as the checker.
 *
 * It restates the reference (phbastosa/FWI2D) in plain C, on the reference's
 * own unpitched layout idx = i + j*nzz (src/modeling/modeling.cu:308-309):
 *   orc_ricker      Ricker samples of set_wavelet             modeling.cu:36-49
 *   orc_b1d         Cerjan profile of set_abc_dampers         modeling.cu:113-150
 *   orc_indices     grid indices of initialization            modeling.cu:252-277
 *   orc_expand      expand_boundary                           modeling.cu:190-218
 *   orc_forward     forward_solver: compute_pressure +
 *                   compute_seismogram per step               modeling.cu:286-353
 *   orc_backward    Migration::backward_propagation /
 *                   Inversion::backward_propagation           migration.cu:61-81,117-180
 *                                                             inversion.cu:230-248,381-444
 *   orc_bumps       set_random_boundary host part +
 *                   poissonDiskSampling                       modeling.cu:431-465, admin.cpp:112-206
 *   orc_rbc         random_boundary_bg + random_boundary_gp   modeling.cu:467-531
 *
 * Compiled twice (oracle/Makefile):
 *   liboracle64.so  REAL = double: every field and sum in FP64 (the FP64 oracle);
 *   liboracle32.so  REAL = float : the reference's own arithmetic - float fields,
 *                   the stencil sums in double because FDM1..5 are double literals
 *                   (modeling.cuh:9-13), the update in float.  OpenMP over columns.
 *
 * Update order (the reference kernels race; this oracle fixes one order):
 * the source is added to P before the stencil reads it, the stencil reads the
 * undamped P of the whole grid, then P and the new field are damped.  With
 * ordered != 0 the points are instead updated one by one in index order with the
 * damping of each point applied at once, which is what a fully serialised run
 * of compute_pressure would see; comparing the two bounds the effect of the
 * reference's in-place damping race.
 *
 * The random boundary uses this project's seeded generator (the reference's is
 * unseeded): SplitMix64 mixing (Steele, Lea & Flood 2014), AS 241 normals
 * (Wichura 1988) and exp/log by range reduction + series, restated here
 * independently of the product so the tests can compare the two bit for bit.
 * Build with -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL double
#endif

#define FDM1 0.001785714285
#define FDM2 0.025396825396
#define FDM3 0.200000000000
#define FDM4 1.600000000000
#define FDM5 2.847222222222

/* ------------------------------------------------------------ set-up ---- */
void orc_ricker(int nt, float dt, float fmax, float* out, int* tlag) {
    float t0 = 2.0f * sqrtf(M_PI) / fmax;
    float fc = fmax / (3.0f * sqrtf(M_PI));
    *tlag = (int)(t0 / dt) + 1;
    for (int n = 0; n < nt; n++) {
        float td = n * dt - t0;
        float arg = M_PI * M_PI * M_PI * fc * fc * td * td;
        out[n] = 1e5f * (1.0f - 2.0f * arg) * expf(-arg);
    }
}

void orc_b1d(int nb, float abc_factor, float* out) {
    for (int i = 0; i < nb; i++) out[i] = expf(-powf(abc_factor * (nb - i), 2.0f));
}

void orc_indices(int n, const float* coord, float dh, int nb, int* out) {
    for (int k = 0; k < n; k++) out[k] = (int)((coord[k] + 0.5f * dh) / dh) + nb;
}

void orc_expand(const float* in, int nz, int nx, int nb, float* out) {
    int nzz = nz + 2 * nb, nxx = nx + 2 * nb;
    for (int j = 0; j < nx; j++)
        for (int i = 0; i < nz; i++) out[(i + nb) + (j + nb) * nzz] = in[i + j * nz];
    for (int i = 0; i < nb; i++)
        for (int j = nb; j < nxx - nb; j++) {
            out[i + j * nzz] = out[nb + j * nzz];
            out[(nzz - i - 1) + j * nzz] = out[(nzz - nb - 1) + j * nzz];
        }
    for (int i = 0; i < nzz; i++)
        for (int j = 0; j < nb; j++) {
            out[i + j * nzz] = out[i + nb * nzz];
            out[i + (nxx - j - 1) * nzz] = out[i + (nxx - nb - 1) * nzz];
        }
}

/* 9-region damper of get_boundary_damper (modeling.cu:355-402) from b1d and
 * b2d = b1d[i] + b1d[j] - 1 built exactly as set_abc_dampers does. */
static float damper(const float* b1d, int nb, int i, int j, int nzz, int nxx) {
    if (i >= nb && i < nzz - nb && j >= nb && j < nxx - nb) return 1.0f;
    if (i < nb && j >= nb && j < nxx - nb) return b1d[i];
    if (i >= nzz - nb && j >= nb && j < nxx - nb) return b1d[nb - (i - (nzz - nb)) - 1];
    if (i >= nb && i < nzz - nb && j < nb) return b1d[j];
    if (i >= nb && i < nzz - nb && j >= nxx - nb) return b1d[nb - (j - (nxx - nb)) - 1];
    int a = (i < nb) ? i : nb - (i - (nzz - nb)) - 1;
    int b = (j < nb) ? j : nb - (j - (nxx - nb)) - 1;
    float s = 0.0f;
    /* b2d[a + b*nb] accumulates b1d[a] and b1d[b]; float + is commutative */
    s += b1d[a];
    s += b1d[b];
    return s - 1.0f;
}

/* d2/dx2 + d2/dz2 of field f at (i, j), in double as the reference evaluates it */
static inline void lap2(const REAL* f, int i, int j, int nzz, float idh2, REAL* dx, REAL* dz) {
    const int b = j * nzz;
    *dx = (REAL)((-FDM1 * (f[i + b - 4 * nzz] + f[i + b + 4 * nzz]) + FDM2 * (f[i + b - 3 * nzz] + f[i + b + 3 * nzz]) -
                  FDM3 * (f[i + b - 2 * nzz] + f[i + b + 2 * nzz]) + FDM4 * (f[i + b - nzz] + f[i + b + nzz]) -
                  FDM5 * (f[i + b])) * idh2);
    *dz = (REAL)((-FDM1 * (f[(i - 4) + b] + f[(i + 4) + b]) + FDM2 * (f[(i - 3) + b] + f[(i + 3) + b]) -
                  FDM3 * (f[(i - 2) + b] + f[(i + 2) + b]) + FDM4 * (f[(i - 1) + b] + f[(i + 1) + b]) -
                  FDM5 * (f[i + b])) * idh2);
}

/* ---------------------------------------------------------- forward ---- */
int orc_forward(const float* vel, int nzz, int nxx, int nb, const float* b1d, const float* wavelet, int nt, int tlag,
                float dt, float dh, int sx, int sz, int nrec, const int* rx, const int* rz, float* seis,
                REAL* p_out, REAL* pold_out, int ordered) {
    const size_t n = (size_t)nzz * nxx;
    REAL* P = (REAL*)calloc(n, sizeof(REAL));
    REAL* Pold = (REAL*)calloc(n, sizeof(REAL));
    if (!P || !Pold) return -1;
    const float idh2 = 1.0f / (dh * dh);
    const int N = nt + tlag;
    for (int t = 0; t < N; t++) {
        if (t < nt) P[sz + sx * nzz] += idh2 * wavelet[t];
        if (!ordered) {
#pragma omp parallel for schedule(static)
            for (int j = 4; j < nxx - 4; j++)
                for (int i = 4; i < nzz - 4; i++) {
                    const size_t idx = (size_t)i + (size_t)j * nzz;
                    const REAL vp2 = (REAL)vel[idx] * (REAL)vel[idx];
                    REAL dx, dz;
                    lap2(P, i, j, nzz, idh2, &dx, &dz);
                    Pold[idx] = (REAL)dt * (REAL)dt * vp2 * (dx + dz) + (REAL)2.0 * P[idx] - Pold[idx];
                }
            if (b1d) {
#pragma omp parallel for schedule(static)
                for (int j = 4; j < nxx - 4; j++)
                    for (int i = 4; i < nzz - 4; i++) {
                        const size_t idx = (size_t)i + (size_t)j * nzz;
                        const float d = damper(b1d, nb, i, j, nzz, nxx);
                        P[idx] *= d;
                        Pold[idx] *= d;
                    }
            }
        } else {
            for (size_t idx = 0; idx < n; idx++) {
                const int i = (int)(idx % nzz), j = (int)(idx / nzz);
                if (!(i > 3 && i < nzz - 4 && j > 3 && j < nxx - 4)) continue;
                const REAL vp2 = (REAL)vel[idx] * (REAL)vel[idx];
                REAL dx, dz;
                lap2(P, i, j, nzz, idh2, &dx, &dz);
                Pold[idx] = (REAL)dt * (REAL)dt * vp2 * (dx + dz) + (REAL)2.0 * P[idx] - Pold[idx];
                if (b1d) {
                    const float d = damper(b1d, nb, i, j, nzz, nxx);
                    P[idx] *= d;
                    Pold[idx] *= d;
                }
            }
        }
        if (seis && t > tlag)
            for (int r = 0; r < nrec; r++) seis[(t - tlag) + (size_t)r * nt] = (float)P[rz[r] + (size_t)rx[r] * nzz];
        REAL* tmp = P;
        P = Pold;
        Pold = tmp;
    }
    if (p_out) memcpy(p_out, P, n * sizeof(REAL));
    if (pold_out) memcpy(pold_out, Pold, n * sizeof(REAL));
    free(P);
    free(Pold);
    return 0;
}

/* --------------------------------------------------------- backward ---- */
/* ps = p^N and psold = p^(N-1) from orc_forward (overwritten).  gradient == 0:
 * acc += Ps_new*Pr (cross_correlation); gradient != 0: acc += dt*Pr*lap*vp^2
 * (build_gradient).  illum += Ps_new^2.  data is nt x nrec trace-major. */
int orc_backward(const float* vel, int nzz, int nxx, const float* data, int nt, int tlag, float dt, float dh, int nrec,
                 const int* rx, const int* rz, REAL* ps, REAL* psold, int gradient, REAL* acc, REAL* illum) {
    const size_t n = (size_t)nzz * nxx;
    REAL* Pr = (REAL*)calloc(n, sizeof(REAL));
    REAL* Prold = (REAL*)calloc(n, sizeof(REAL));
    if (!Pr || !Prold) return -1;
    const float idh2 = 1.0f / (dh * dh);
    REAL* Ps = ps;
    REAL* Psold = psold;
    const int N = nt + tlag;
    for (int t = 0; t < N; t++) {
        if (t < nt)
            for (int r = 0; r < nrec; r++) Pr[rz[r] + (size_t)rx[r] * nzz] += idh2 * data[(nt - t - 1) + (size_t)r * nt];
#pragma omp parallel for schedule(static)
        for (int j = 4; j < nxx - 4; j++)
            for (int i = 4; i < nzz - 4; i++) {
                const size_t idx = (size_t)i + (size_t)j * nzz;
                const REAL vp2 = (REAL)vel[idx] * (REAL)vel[idx];
                REAL sx, sz, rxx, rzz;
                lap2(Psold, i, j, nzz, idh2, &sx, &sz);
                lap2(Pr, i, j, nzz, idh2, &rxx, &rzz);
                Ps[idx] = (REAL)dt * (REAL)dt * vp2 * (sx + sz) + (REAL)2.0 * Psold[idx] - Ps[idx];
                Prold[idx] = (REAL)dt * (REAL)dt * vp2 * (rxx + rzz) + (REAL)2.0 * Pr[idx] - Prold[idx];
                illum[idx] += Ps[idx] * Ps[idx];
                if (gradient) acc[idx] += (REAL)dt * Pr[idx] * (sx + sz) * vp2;
                else acc[idx] += Ps[idx] * Pr[idx];
            }
        REAL* tmp = Ps;
        Ps = Psold;
        Psold = tmp;
        tmp = Pr;
        Pr = Prold;
        Prold = tmp;
    }
    free(Pr);
    free(Prold);
    return 0;
}

/* ---------------------------------------------- seeded generator ------- */
static uint64_t o_mix(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static uint64_t o_key(uint64_t seed, uint32_t shot, uint32_t stream) {
    return o_mix(o_mix(seed) ^ (((uint64_t)shot << 32) | (uint64_t)stream));
}
static uint64_t o_draw(uint64_t key, uint64_t ctr) { return o_mix(key ^ o_mix(ctr)); }
static float o_u01f(uint64_t h) { return (float)(uint32_t)(h >> 40) * 5.9604644775390625e-8f; }

static double o_from_bits(uint64_t b) { double d; memcpy(&d, &b, 8); return d; }
static uint64_t o_to_bits(double d) { uint64_t b; memcpy(&b, &d, 8); return b; }

static double o_log(double x) {  /* x > 0, normal */
    uint64_t b = o_to_bits(x);
    int e = (int)((b >> 52) & 0x7FF) - 1023;
    double m = o_from_bits((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
    if (m > 1.4142135623730951) { m = m * 0.5; e = e + 1; }
    double s = (m - 1.0) / (m + 1.0), s2 = s * s;
    static const double inv_odd[] = {1.0 / 23.0, 1.0 / 21.0, 1.0 / 19.0, 1.0 / 17.0, 1.0 / 15.0, 1.0 / 13.0,
                                     1.0 / 11.0, 1.0 / 9.0,  1.0 / 7.0,  1.0 / 5.0,  1.0 / 3.0,  1.0};
    double p = inv_odd[0];
    for (int k = 1; k < 12; k++) p = p * s2 + inv_odd[k];
    double lm = 2.0 * s * p;
    return ((double)e * 6.93147180369123816490e-01 + lm) + (double)e * 1.90821492927058770002e-10;
}

static double o_exp(double x) {  /* x <= 0 */
    if (x < -708.0) return 0.0;
    double kf = x * 1.44269504088896338700e+00 + 0.5;
    int k = (int)kf;
    if ((double)k > kf) k = k - 1;
    double r = (x - (double)k * 6.93147180369123816490e-01) - (double)k * 1.90821492927058770002e-10;
    static const double inv_fact[] = {1.0 / 6227020800.0, 1.0 / 479001600.0, 1.0 / 39916800.0, 1.0 / 3628800.0,
                                      1.0 / 362880.0,     1.0 / 40320.0,     1.0 / 5040.0,     1.0 / 720.0,
                                      1.0 / 120.0,        1.0 / 24.0,        1.0 / 6.0,        0.5,
                                      1.0,                1.0};
    double p = inv_fact[0];
    for (int q = 1; q < 14; q++) p = p * r + inv_fact[q];
    if (k < -1022) {
        p = p * o_from_bits((uint64_t)(k + 600 + 1023) << 52);
        return p * o_from_bits((uint64_t)(-600 + 1023) << 52);
    }
    return p * o_from_bits((uint64_t)(k + 1023) << 52);
}

static double o_poly(const double* c, int n, double r) { /* c[0]*r^(n-1) + ... + c[n-1], Horner */
    double p = c[0];
    for (int k = 1; k < n; k++) p = p * r + c[k];
    return p;
}

/* AS 241 PPND16 */
static double o_ppnd16(double p) {
    static const double A[] = {2.5090809287301226727e+3, 3.3430575583588128105e+4, 6.7265770927008700853e+4,
                               4.5921953931549871457e+4, 1.3731693765509461125e+4, 1.9715909503065514427e+3,
                               1.3314166789178437745e+2, 3.3871328727963666080e0};
    static const double B[] = {5.2264952788528545610e+3, 2.8729085735721942674e+4, 3.9307895800092710610e+4,
                               2.1213794301586595867e+4, 5.3941960214247511077e+3, 6.8718700749205790830e+2,
                               4.2313330701600911252e+1, 1.0};
    static const double C[] = {7.74545014278341407640e-4, 2.27238449892691845833e-2, 2.41780725177450611770e-1,
                               1.27045825245236838258e0,  3.64784832476320460504e0,  5.76949722146069140550e0,
                               4.63033784615654529590e0,  1.42343711074968357734e0};
    static const double D[] = {1.05075007164441684324e-9, 5.47593808499534494600e-4, 1.51986665636164571966e-2,
                               1.48103976427480074590e-1, 6.89767334985100004550e-1, 1.67638483018380384940e0,
                               2.05319162663775882187e0,  1.0};
    static const double E[] = {2.01033439929228813265e-7, 2.71155556874348757815e-5, 1.24266094738807843860e-3,
                               2.65321895265761230930e-2, 2.96560571828504891230e-1, 1.78482653991729133580e0,
                               5.46378491116411436990e0,  6.65790464350110377720e0};
    static const double F[] = {2.04426310338993978564e-15, 1.42151175831644588870e-7, 1.84631831751005468180e-5,
                               7.86869131145613259100e-4,  1.48753612908506148525e-2, 1.36929880922735805310e-1,
                               5.99832206555887937690e-1,  1.0};
    double q = p - 0.5;
    if (fabs(q) <= 0.425) {
        double r = 0.180625 - q * q;
        return q * o_poly(A, 8, r) / o_poly(B, 8, r);
    }
    double r = q < 0 ? p : 1.0 - p;
    r = sqrt(-o_log(r));
    double v;
    if (r <= 5.0) { r = r - 1.6; v = o_poly(C, 8, r) / o_poly(D, 8, r); }
    else { r = r - 5.0; v = o_poly(E, 8, r) / o_poly(F, 8, r); }
    return q < 0 ? -v : v;
}

static float o_normal(uint64_t key, uint64_t ctr) {
    uint64_t h = o_draw(key, ctr);
    double u = ((double)(h >> 11) + 0.5) * 1.1102230246251565e-16;
    return (float)o_ppnd16(u);
}

/* exported for the generator tests */
double orc_ppnd16(double p) { return o_ppnd16(p); }
double orc_exp(double x) { return o_exp(x); }
double orc_log(double x) { return o_log(x); }
float orc_normal(uint64_t seed, uint32_t shot, uint32_t stream, uint64_t ctr) {
    return o_normal(o_key(seed, shot, stream), ctr);
}

/* ------------------------------------------------ random boundary ------ */
typedef struct { float x, z; } OPt;
typedef struct { uint64_t key, ctr; } OStream;
static uint64_t os_next(OStream* s) { return o_draw(s->key, s->ctr++); }
static float os_uniform(OStream* s, float a, float b) { return a + (b - a) * o_u01f(os_next(s)); }

/* Bridson sampling (30 tries per active point) of [0,x_max) x [0,z_max) with
 * the structure of poissonDiskSampling; returns the number of points written
 * to out (at most cap). */
static int o_pds(float x_max, float z_max, float radius, uint64_t seed, uint32_t shot, OPt* out, int cap) {
    OStream rng = {o_key(seed, shot, 3u), 0};
    const float cell = radius / sqrtf(2.0f);
    const int gx_n = (int)ceilf(x_max / cell), gz_n = (int)ceilf(z_max / cell);
    OPt* grid = (OPt*)malloc(sizeof(OPt) * (size_t)gx_n * gz_n);
    OPt* active = (OPt*)malloc(sizeof(OPt) * (size_t)(cap > 0 ? cap : 1));
    for (size_t k = 0; k < (size_t)gx_n * gz_n; k++) { grid[k].x = -1.0f; grid[k].z = -1.0f; }
    int np = 0, na = 0;
    const float two_pi = (float)(2.0 * M_PI);
    OPt p0;
    p0.x = os_uniform(&rng, 0.0f, x_max);
    p0.z = os_uniform(&rng, 0.0f, z_max);
    out[np++] = p0;
    active[na++] = p0;
    grid[(size_t)(int)(p0.z / cell) + (size_t)(int)(p0.x / cell) * gz_n] = p0;
    while (na > 0) {
        int idx = (int)((os_next(&rng) >> 11) % (uint64_t)na);
        OPt base = active[idx];
        int found = 0;
        for (int t = 0; t < 30; t++) {
            float ang = os_uniform(&rng, 0.0f, two_pi);
            float r = os_uniform(&rng, radius, 2.0f * radius);
            OPt q;
            q.x = base.x + r * cosf(ang);
            q.z = base.z + r * sinf(ang);
            int ok = !(q.x < 0 || q.z < 0 || q.x >= x_max || q.z >= z_max);
            if (ok) {
                int gx = (int)(q.x / cell), gz = (int)(q.z / cell);
                for (int di = -1; di <= 1 && ok; di++)
                    for (int dj = -1; dj <= 1 && ok; dj++) {
                        int nx = gx + dj, nz = gz + di;
                        if (nx >= 0 && nz >= 0 && nx < gx_n && nz < gz_n) {
                            OPt nb = grid[(size_t)nz + (size_t)nx * gz_n];
                            float dx = nb.x - q.x, dz = nb.z - q.z;
                            if (nb.x != -1.0f && sqrtf(dx * dx + dz * dz) < radius) ok = 0;
                        }
                    }
            }
            if (ok && np < cap) {
                out[np++] = q;
                active[na++] = q;
                grid[(size_t)(int)(q.z / cell) + (size_t)(int)(q.x / cell) * gz_n] = q;
                found = 1;
            }
        }
        if (!found) {
            memmove(active + idx, active + idx + 1, sizeof(OPt) * (size_t)(na - idx - 1));
            na--;
        }
    }
    free(grid);
    free(active);
    return np;
}

/* The raw point set of one shot's sampler, before the band filter of
 * set_random_boundary: (x, z) pairs into out; returns the count (at most cap
 * are written). */
int orc_pds(float x_max, float z_max, float radius, uint64_t seed, uint32_t shot, float* out, int cap) {
    OPt* pts = (OPt*)malloc(sizeof(OPt) * (size_t)(cap > 0 ? cap : 1));
    int np = o_pds(x_max, z_max, radius, seed, shot, pts, cap);
    for (int k = 0; k < np && k < cap; k++) { out[2 * k] = pts[k].x; out[2 * k + 1] = pts[k].z; }
    free(pts);
    return np;
}

/* Bumps of one shot: (xc, zc, r, A, factor) x count into out (5 floats each). */
int orc_bumps(int nxx, int nzz, int nb, float dh, float ratio, float varVp, uint64_t seed, uint32_t shot,
              float* out, int cap) {
    float x_max = (nxx - 1) * dh, z_max = (nzz - 1) * dh;
    int pcap = 1 << 20;
    OPt* pts = (OPt*)malloc(sizeof(OPt) * (size_t)pcap);
    int np = o_pds(x_max, z_max, ratio, seed, shot, pts, pcap);
    float fnb = (float)nb * dh;
    OStream rng = {o_key(seed, shot, 4u), 0};
    int nbump = 0;
    for (int k = 0; k < np; k++) {
        OPt p = pts[k];
        if ((p.x > 0.5f * fnb) && (p.x < x_max - 0.5f * fnb) && (p.z > 0.5f * fnb) && (p.z < z_max - 0.5f * fnb)) continue;
        float r = os_uniform(&rng, 0.2f * ratio, ratio);
        float A = os_uniform(&rng, 0.5f * varVp, varVp);
        float factor = (os_next(&rng) % 3 == 0) ? 1.0f : -1.0f;
        if (nbump < cap) {
            float* o = out + 5 * (size_t)nbump;
            o[0] = p.x; o[1] = p.z; o[2] = r; o[3] = A; o[4] = factor;
        }
        nbump++;
    }
    free(pts);
    return nbump;
}

/* random_boundary_bg then every bump (random_boundary_gp) on the padded,
 * edge-replicated velocity `base`; result in out (both nzz x nxx). */
void orc_rbc(const float* base, int nzz, int nxx, int nb, float dh, float varVp, float vmin, float vmax,
             uint64_t seed, uint32_t shot, const float* bumps, int nbump, float* out) {
    const uint64_t kx = o_key(seed, shot, 1u), kz = o_key(seed, shot, 2u);
    memcpy(out, base, sizeof(float) * (size_t)nzz * nxx);
    /* random_boundary_bg */
    for (int j = 0; j < nxx; j++)
        for (int i = 0; i < nzz; i++) {
            if (i >= nb && i < nzz - nb && j >= nb && j < nxx - nb) continue;
            int ii = i < nb ? nb : (i > nzz - nb - 1 ? nzz - nb - 1 : i);
            int jj = j < nb ? nb : (j > nxx - nb - 1 ? nxx - nb - 1 : j);
            float val = base[ii + (size_t)jj * nzz];
            uint64_t idx = (uint64_t)i + (uint64_t)j * nzz;
            if (j < nb) {
                float fx = 1.0f - (float)(j) / (float)(nb);
                val = val + fx * varVp * o_normal(kx, idx);
            } else if (j >= nxx - nb) {
                float fx = 1.0f - (float)(nxx - j - 1) / (float)(nb);
                val = val + fx * varVp * o_normal(kx, idx);
            }
            if (i < nb) {
                float fz = 1.0f - (float)(i) / (float)(nb);
                val = val + fz * varVp * o_normal(kz, idx);
            } else if (i >= nzz - nb) {
                float fz = 1.0f - (float)(nzz - i - 1) / (float)(nb);
                val = val + fz * varVp * o_normal(kz, idx);
            }
            out[i + (size_t)j * nzz] = val;
        }
    /* random_boundary_gp, one pass per bump as the reference launches them */
    const float x_max = (nxx - 1) * dh, z_max = (nzz - 1) * dh, fnb = (float)(nb) * dh;
    for (int p = 0; p < nbump; p++) {
        const float xc = bumps[5 * p], zc = bumps[5 * p + 1], r = bumps[5 * p + 2], A = bumps[5 * p + 3],
                    factor = bumps[5 * p + 4];
        for (int j = 0; j < nxx; j++) {
            const float X = (float)(j) * dh;
            for (int i = 0; i < nzz; i++) {
                const float Z = (float)(i) * dh;
                if ((X > fnb) && (X < x_max - fnb) && (Z > fnb) && (Z < z_max - fnb)) continue;
                float v = out[i + (size_t)j * nzz];
                float ax = (X - xc) / r, az = (Z - zc) / r;
                v += factor * A * (float)o_exp((double)(-0.5f * (ax * ax + az * az)));
                v = v > vmax + varVp ? vmax + varVp : v;
                v = v < vmin - varVp ? vmin - varVp : v;
                out[i + (size_t)j * nzz] = v;
            }
        }
    }
}
