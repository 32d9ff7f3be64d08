/*
 * clg_oracle_measure.c -- FP64 CPU restatement of CLGLib's measurement
 * contractions on top of the fermion solves.
 *
 * TEST INFRASTRUCTURE ONLY (the checker): the product library never links it.
 *
 *  - the chiral gamma-matrix set and its products (Tools/Math/GammaMatrix.h:
 *    gammaMatrixSet::CreateGammaMatrix :405-511, _mult / _mult_i :293-330,
 *    CalculateNextSymmetricIndex :348-379), indexed by EGammaMatrix
 *    (Core/CudaHelper.h:37-63);
 *  - the meson correlator of 12 point-source propagators
 *    (_kernelCalculateCorrelatorSU3, Measurement/CMeasureMesonCorrelator.cu:26-174,
 *    spatial sums times 2/sqrt(V) :366-380);
 *  - the stochastic condensate traces eta^+ Gamma psi / V
 *    (_kernelDotMeasureAll, Measurement/CMeasureChiralCondensate.cu:38-100).
 */
#include <complex.h>
#include <math.h>
#include <string.h>

#include "clg_oracle.h"

typedef double _Complex cplx;

typedef struct {
    int idx[4]; /* row r has its non-zero entry in column idx[r] ... */
    int z[4];   /* ... equal to i^z[r] */
} gm_t;

static void gm_set(gm_t* g, int r, int c, int z) { g->idx[r] = c, g->z[r] = z; }

/* (a b)_{rc}: row r of a picks row idx_a[r] of b */
static gm_t gm_mult(const gm_t* a, const gm_t* b, int extra_i) {
    gm_t o;
    for (int r = 0; r < 4; ++r) {
        o.idx[r] = b->idx[a->idx[r]];
        o.z[r] = (a->z[r] + b->z[a->idx[r]] + extra_i) & 3;
    }
    return o;
}

int clgo_gamma(int which, int idx[4], int z[4], int* next_symmetric) {
    if (which < 0 || which >= CLGO_EGM_MAX) return -1;
    gm_t g[CLGO_EGM_MAX];
    memset(g, 0, sizeof g);
    for (int r = 0; r < 4; ++r) gm_set(&g[CLGO_UNITY], r, r, 0);
    /* chiral set */
    gm_set(&g[CLGO_GAMMA1], 0, 3, 3), gm_set(&g[CLGO_GAMMA1], 1, 2, 3), gm_set(&g[CLGO_GAMMA1], 2, 1, 1),
        gm_set(&g[CLGO_GAMMA1], 3, 0, 1);
    gm_set(&g[CLGO_GAMMA2], 0, 3, 2), gm_set(&g[CLGO_GAMMA2], 1, 2, 0), gm_set(&g[CLGO_GAMMA2], 2, 1, 0),
        gm_set(&g[CLGO_GAMMA2], 3, 0, 2);
    gm_set(&g[CLGO_GAMMA3], 0, 2, 3), gm_set(&g[CLGO_GAMMA3], 1, 3, 1), gm_set(&g[CLGO_GAMMA3], 2, 0, 1),
        gm_set(&g[CLGO_GAMMA3], 3, 1, 3);
    gm_set(&g[CLGO_GAMMA4], 0, 2, 0), gm_set(&g[CLGO_GAMMA4], 1, 3, 0), gm_set(&g[CLGO_GAMMA4], 2, 0, 0),
        gm_set(&g[CLGO_GAMMA4], 3, 1, 0);
    gm_set(&g[CLGO_GAMMA5], 0, 0, 0), gm_set(&g[CLGO_GAMMA5], 1, 1, 0), gm_set(&g[CLGO_GAMMA5], 2, 2, 2),
        gm_set(&g[CLGO_GAMMA5], 3, 3, 2);
    g[CLGO_GAMMA51] = gm_mult(&g[CLGO_GAMMA5], &g[CLGO_GAMMA1], 0);
    g[CLGO_GAMMA52] = gm_mult(&g[CLGO_GAMMA5], &g[CLGO_GAMMA2], 0);
    g[CLGO_GAMMA53] = gm_mult(&g[CLGO_GAMMA5], &g[CLGO_GAMMA3], 0);
    g[CLGO_GAMMA54] = gm_mult(&g[CLGO_GAMMA5], &g[CLGO_GAMMA4], 0);
    g[CLGO_GAMMA15] = gm_mult(&g[CLGO_GAMMA1], &g[CLGO_GAMMA5], 0);
    g[CLGO_GAMMA25] = gm_mult(&g[CLGO_GAMMA2], &g[CLGO_GAMMA5], 0);
    g[CLGO_GAMMA35] = gm_mult(&g[CLGO_GAMMA3], &g[CLGO_GAMMA5], 0);
    g[CLGO_GAMMA45] = gm_mult(&g[CLGO_GAMMA4], &g[CLGO_GAMMA5], 0);
    g[CLGO_SIGMA12] = gm_mult(&g[CLGO_GAMMA2], &g[CLGO_GAMMA1], 1);
    g[CLGO_SIGMA23] = gm_mult(&g[CLGO_GAMMA3], &g[CLGO_GAMMA2], 1);
    g[CLGO_SIGMA31] = gm_mult(&g[CLGO_GAMMA1], &g[CLGO_GAMMA3], 1);
    g[CLGO_SIGMA12E] = gm_mult(&g[CLGO_GAMMA1], &g[CLGO_GAMMA2], 1);
    g[CLGO_SIGMA23E] = gm_mult(&g[CLGO_GAMMA2], &g[CLGO_GAMMA3], 1);
    g[CLGO_SIGMA31E] = gm_mult(&g[CLGO_GAMMA3], &g[CLGO_GAMMA1], 1);
    g[CLGO_SIGMA41] = gm_mult(&g[CLGO_GAMMA1], &g[CLGO_GAMMA4], 1);
    g[CLGO_SIGMA42] = gm_mult(&g[CLGO_GAMMA2], &g[CLGO_GAMMA4], 1);
    g[CLGO_SIGMA43] = gm_mult(&g[CLGO_GAMMA3], &g[CLGO_GAMMA4], 1);
    g[CLGO_CHARGECONJG] = gm_mult(&g[CLGO_GAMMA4], &g[CLGO_GAMMA2], 0);
    for (int r = 0; r < 4; ++r) idx[r] = g[which].idx[r], z[r] = g[which].z[r];
    /* CalculateNextSymmetricIndex: 0 -> 0, 1 -> 2, 2 -> 3, 3 -> 1 by idx[0] */
    static const int nsi[4] = {0, 2, 3, 1};
    *next_symmetric = nsi[g[which].idx[0]];
    return 0;
}

/* S(j, a)[s]_{i, b}: sink spin i colour b at site s of the propagator of source spin j colour a */
static inline cplx prop_at(const double* prop, long V, int j, int a, long s, int i, int b) {
    const double* p = prop + ((long)(3 * j + a) * V + s) * 24 + 2 * (3 * i + b);
    return p[0] + I * p[1];
}

/* sum_{a, b} Re(conj(S(j,a)_{i,b}) S(pj,a)_{pi,b}) */
static double meson_term(const double* prop, long V, long s, int i, int j, int pi, int pj) {
    double t = 0.0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) t += creal(conj(prop_at(prop, V, j, a, s, i, b)) * prop_at(prop, V, pj, a, s, pi, b));
    return t;
}

void clgo_meson_correlator(const int L[4], const double* prop, int gamma, double* C) {
    int idx[4], z[4], ns;
    clgo_gamma(gamma, idx, z, &ns);
    const long V = (long)L[0] * L[1] * L[2] * L[3];
    const int Lt = L[3];
    for (int t = 0; t < Lt; ++t) C[t] = 0.0;
    for (long s = 0; s < V; ++s) {
        double res = 0.0;
        for (int i = 1; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j) {
                /* c1 c2^*: i^(z_i + conj(z_j)), conj(i^b) = i^(((b & 1) << 1) + b) */
                const int zz = z[i] + (((z[j] & 1) << 1) + z[j]);
                res += (1.0 - (double)(zz & 2)) * meson_term(prop, V, s, i, j, idx[i], idx[j]);
            }
        if (ns == 0) {
            for (int i = 0; i < 4; ++i) res += 0.5 * meson_term(prop, V, s, i, i, i, i);
        } else {
            res += meson_term(prop, V, s, 0, 0, idx[0], idx[0]);
            res += meson_term(prop, V, s, ns, ns, idx[ns], idx[ns]);
        }
        C[s % Lt] += res;
    }
    const double f = 2.0 / sqrt((double)V);
    for (int t = 0; t < Lt; ++t) C[t] *= f;
}

void clgo_condensate(long V, const double* eta, const double* psi, int kind, double* re_im) {
    int g;
    switch (kind) {
        case 1: case 2: case 3: case 4: case 5: g = kind; break;
        case 6: g = CLGO_GAMMA45; break;
        case 7: g = CLGO_GAMMA1; break; /* gamma1 + y omega gamma4 at omega = 0 */
        case 8: g = CLGO_GAMMA2; break; /* gamma2 - x omega gamma4 at omega = 0 */
        default: g = CLGO_UNITY; break;
    }
    int idx[4], z[4], ns;
    clgo_gamma(g, idx, z, &ns);
    static const double zr[4] = {1, 0, -1, 0}, zi[4] = {0, 1, 0, -1};
    cplx acc = 0.0;
    for (long s = 0; s < V; ++s)
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 3; ++c) {
                const double* e = eta + s * 24 + 2 * (3 * r + c);
                const double* q = psi + s * 24 + 2 * (3 * idx[r] + c);
                const cplx gp = (zr[z[r]] + I * zi[z[r]]) * (q[0] + I * q[1]);
                acc += conj(e[0] + I * e[1]) * gp;
            }
    acc /= (double)V;
    re_im[0] = creal(acc);
    re_im[1] = cimag(acc);
}
