/*
 * clg_oracle_fields.c -- seeded synthetic fields, the plaquette and the
 * Bridge++ reorder, restated on the CPU in FP64.
 *
 * TEST INFRASTRUCTURE ONLY.  The product library carries its own (device)
 * generator; the tests compare the two.
 *
 * Generator (published methods, written here from the papers):
 *   - Philox4x32-10 counter-based RNG: J. Salmon, M. Moraes, R. Dror,
 *     D. Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11.
 *     key = {seed_lo32, seed_hi32 ^ field_id}; counter = {index_lo, index_hi, sub, tag}.
 *   - Gaussians by Box-Muller from two 53-bit uniforms in (0,1).
 *   - Complex Gaussian with E|z|^2 = 1 (re, im ~ N(0, 1/2)), the reference's
 *     convention (Tools/Math/Random.h:188-197).
 *   - Haar SU(3): QR of a complex-Gaussian 3x3 with the R diagonal made
 *     positive (Gram-Schmidt on columns, F. Mezzadri, "How to generate random
 *     matrices from the classical compact groups", Notices AMS 54 (2007)),
 *     then column 2 multiplied by conj(det) so det = 1.
 *   - exp(i eps H), H = sum_a h_a lambda_a / 2 with h_a ~ N(0,1) (Gell-Mann
 *     lambda_a): Taylor series with scaling and squaring in FP64, then
 *     re-unitarised (rows 0,1 Gram-Schmidt, row 2 = conj(row0 x row1)).
 */
#include "clg_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex cplx;

enum { TAG_GAUGE = 0x47415547u, TAG_SPINOR = 0x5350494eu, TAG_Z2 = 0x5a324e53u, TAG_Z4 = 0x5a344e53u };

void clgo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline double u53(uint32_t a, uint32_t b) {
    const uint64_t x = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);
    return ((double)x + 0.5) * (1.0 / 9007199254740992.0);
}

/* two N(0,1) from one Philox call */
static inline void gauss2(uint64_t seed, uint32_t field_id, uint64_t index, uint32_t sub, uint32_t tag,
                          double* g1, double* g2) {
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32) ^ field_id};
    const uint32_t ctr[4] = {(uint32_t)index, (uint32_t)(index >> 32), sub, tag};
    uint32_t o[4];
    clgo_philox4x32_10(ctr, key, o);
    const double u1 = u53(o[0], o[1]);
    const double u2 = u53(o[2], o[3]);
    const double r = sqrt(-2.0 * log(u1));
    const double th = 6.283185307179586476925286766559 * u2;
    *g1 = r * cos(th);
    *g2 = r * sin(th);
}

static void haar_su3(uint64_t seed, uint32_t field_id, uint64_t link, cplx m[9]) {
    const double isq2 = 0.70710678118654752440084436210485;
    cplx z[9];
    for (int k = 0; k < 9; ++k) {
        double a, b;
        gauss2(seed, field_id, link, (uint32_t)k, TAG_GAUGE, &a, &b);
        z[k] = (a + I * b) * isq2;
    }
    /* Gram-Schmidt on columns */
    for (int c = 0; c < 3; ++c) {
        for (int p = 0; p < c; ++p) {
            cplx d = 0;
            for (int r = 0; r < 3; ++r) d += conj(z[3 * r + p]) * z[3 * r + c];
            for (int r = 0; r < 3; ++r) z[3 * r + c] -= d * z[3 * r + p];
        }
        double nn = 0;
        for (int r = 0; r < 3; ++r) nn += creal(z[3 * r + c] * conj(z[3 * r + c]));
        const double inv = 1.0 / sqrt(nn);
        for (int r = 0; r < 3; ++r) z[3 * r + c] *= inv;
    }
    const cplx det = z[0] * (z[4] * z[8] - z[5] * z[7]) - z[1] * (z[3] * z[8] - z[5] * z[6]) +
                     z[2] * (z[3] * z[7] - z[4] * z[6]);
    const cplx f = conj(det);
    for (int r = 0; r < 3; ++r) z[3 * r + 2] *= f;
    memcpy(m, z, sizeof(cplx) * 9);
}

static void reunitarise(cplx m[9]) {
    /* row 0 */
    double n0 = 0;
    for (int k = 0; k < 3; ++k) n0 += creal(m[k] * conj(m[k]));
    n0 = 1.0 / sqrt(n0);
    for (int k = 0; k < 3; ++k) m[k] *= n0;
    /* row 1 orthogonal to row 0 */
    cplx d = 0;
    for (int k = 0; k < 3; ++k) d += conj(m[k]) * m[3 + k];
    for (int k = 0; k < 3; ++k) m[3 + k] -= d * m[k];
    double n1 = 0;
    for (int k = 0; k < 3; ++k) n1 += creal(m[3 + k] * conj(m[3 + k]));
    n1 = 1.0 / sqrt(n1);
    for (int k = 0; k < 3; ++k) m[3 + k] *= n1;
    /* row 2 = conj(row0 x row1) */
    m[6] = conj(m[1] * m[5] - m[2] * m[4]);
    m[7] = conj(m[2] * m[3] - m[0] * m[5]);
    m[8] = conj(m[0] * m[4] - m[1] * m[3]);
}

static void expH_su3(uint64_t seed, uint32_t field_id, uint64_t link, double eps, cplx m[9]) {
    double h[8];
    for (int k = 0; k < 4; ++k) gauss2(seed, field_id, link, (uint32_t)k, TAG_GAUGE, &h[2 * k], &h[2 * k + 1]);
    const double is3 = 0.57735026918962576450914878050196;
    /* H = sum_a h_a lambda_a / 2 */
    cplx H[9];
    H[0] = 0.5 * (h[2] + h[7] * is3);
    H[4] = 0.5 * (-h[2] + h[7] * is3);
    H[8] = 0.5 * (-2.0 * h[7] * is3);
    H[1] = 0.5 * (h[0] - I * h[1]);
    H[3] = conj(H[1]);
    H[2] = 0.5 * (h[3] - I * h[4]);
    H[6] = conj(H[2]);
    H[5] = 0.5 * (h[5] - I * h[6]);
    H[7] = conj(H[5]);
    /* A = i eps H */
    cplx A[9];
    double fn = 0;
    for (int k = 0; k < 9; ++k) { A[k] = I * eps * H[k]; fn += creal(A[k] * conj(A[k])); }
    fn = sqrt(fn);
    int s = 0;
    while (fn > 0.25) { fn *= 0.5; ++s; }
    const double scale = ldexp(1.0, -s);
    for (int k = 0; k < 9; ++k) A[k] *= scale;
    /* Taylor: E = sum_{k=0}^{18} A^k / k!  (Horner) */
    cplx E[9], T[9];
    for (int k = 0; k < 9; ++k) E[k] = (k % 4 == 0) ? 1.0 : 0.0;
    for (int n = 18; n >= 1; --n) {
        /* E = 1 + A E / n */
        cplx P[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                P[3 * r + c] = A[3 * r] * E[c] + A[3 * r + 1] * E[3 + c] + A[3 * r + 2] * E[6 + c];
        for (int k = 0; k < 9; ++k) E[k] = ((k % 4 == 0) ? 1.0 : 0.0) + P[k] / (double)n;
    }
    for (int q = 0; q < s; ++q) {
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                T[3 * r + c] = E[3 * r] * E[c] + E[3 * r + 1] * E[3 + c] + E[3 * r + 2] * E[6 + c];
        memcpy(E, T, sizeof(E));
    }
    reunitarise(E);
    memcpy(m, E, sizeof(cplx) * 9);
}

static inline long volume(const int L[4]) { return (long)L[0] * L[1] * L[2] * L[3]; }

static void store(double* U, long link, const cplx m[9]) {
    for (int k = 0; k < 9; ++k) { U[18 * link + 2 * k] = creal(m[k]); U[18 * link + 2 * k + 1] = cimag(m[k]); }
}
static void load(const double* U, long link, cplx m[9]) {
    for (int k = 0; k < 9; ++k) m[k] = U[18 * link + 2 * k] + I * U[18 * link + 2 * k + 1];
}

void clgo_gen_gauge_haar(const int L[4], uint64_t seed, uint32_t field_id, double* U) {
    const long nl = volume(L) * 4;
#pragma omp parallel for schedule(static)
    for (long l = 0; l < nl; ++l) {
        cplx m[9];
        haar_su3(seed, field_id, (uint64_t)l, m);
        store(U, l, m);
    }
}

void clgo_gen_gauge_expH(const int L[4], uint64_t seed, uint32_t field_id, double eps, double* U) {
    const long nl = volume(L) * 4;
#pragma omp parallel for schedule(static)
    for (long l = 0; l < nl; ++l) {
        cplx m[9];
        expH_su3(seed, field_id, (uint64_t)l, eps, m);
        store(U, l, m);
    }
}

void clgo_gen_gauge_identity(const int L[4], double* U) {
    const long nl = volume(L) * 4;
    memset(U, 0, sizeof(double) * 18 * nl);
    for (long l = 0; l < nl; ++l) { U[18 * l] = 1.0; U[18 * l + 8] = 1.0; U[18 * l + 16] = 1.0; }
}

/* complex Gaussian spinor, E|z|^2 = 1 per component; one Philox call per component */
void clgo_gen_gauss(long nsites, int ncomp, uint64_t seed, uint32_t field_id, double* psi) {
    const double isq2 = 0.70710678118654752440084436210485;
#pragma omp parallel for schedule(static)
    for (long s = 0; s < nsites; ++s)
        for (int k = 0; k < ncomp; ++k) {
            double a, b;
            gauss2(seed, field_id, (uint64_t)s, (uint32_t)k, TAG_SPINOR, &a, &b);
            psi[2 * (s * ncomp + k)] = a * isq2;
            psi[2 * (s * ncomp + k) + 1] = b * isq2;
        }
}

/* Z2 noise (+-1 +- i)/sqrt(2): bits 2k, 2k+1 of one 128-bit Philox output per site
 * (ncomp <= 64). */
void clgo_gen_z2(long nsites, int ncomp, uint64_t seed, uint32_t field_id, double* psi) {
    const double isq2 = 0.70710678118654752440084436210485;
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32) ^ field_id};
#pragma omp parallel for schedule(static)
    for (long s = 0; s < nsites; ++s) {
        const uint32_t ctr[4] = {(uint32_t)s, (uint32_t)((uint64_t)s >> 32), 0u, TAG_Z2};
        uint32_t o[4];
        clgo_philox4x32_10(ctr, key, o);
        for (int k = 0; k < ncomp; ++k) {
            const int b0 = 2 * k, b1 = 2 * k + 1;
            const uint32_t w0 = o[b0 >> 5] >> (b0 & 31), w1 = o[b1 >> 5] >> (b1 & 31);
            psi[2 * (s * ncomp + k)] = (w0 & 1u) ? -isq2 : isq2;
            psi[2 * (s * ncomp + k) + 1] = (w1 & 1u) ? -isq2 : isq2;
        }
    }
}

/* Z4 noise i^b per component (EFIT_RandomZ4, Tools/Math/Random.h:199-220), b =
 * bits 2k, 2k+1 of one 128-bit Philox output per site (ncomp <= 64). */
void clgo_gen_z4(long nsites, int ncomp, uint64_t seed, uint32_t field_id, double* psi) {
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32) ^ field_id};
#pragma omp parallel for schedule(static)
    for (long s = 0; s < nsites; ++s) {
        const uint32_t ctr[4] = {(uint32_t)s, (uint32_t)((uint64_t)s >> 32), 0u, TAG_Z4};
        uint32_t o[4];
        clgo_philox4x32_10(ctr, key, o);
        for (int k = 0; k < ncomp; ++k) {
            const uint32_t b = (o[(2 * k) >> 5] >> ((2 * k) & 31)) & 3u;
            psi[2 * (s * ncomp + k)] = b == 0 ? 1.0 : (b == 2 ? -1.0 : 0.0);
            psi[2 * (s * ncomp + k) + 1] = b == 1 ? 1.0 : (b == 3 ? -1.0 : 0.0);
        }
    }
}

/* spin-colour point source (CFieldFermionWilsonSquareSU3.cu:521-566, :1222-1255) */
void clgo_gen_point(long nsites, int ncomp, long site, int comp, double* psi) {
    memset(psi, 0, sizeof(double) * 2 * nsites * ncomp);
    psi[2 * (site * ncomp + comp)] = 1.0;
}

void clgo_zero_parity(const int L[4], int ncomp, int parity, double* psi) {
    const long V = volume(L);
    for (long s = 0; s < V; ++s) {
        long t = s;
        int c3 = (int)(t % L[3]); t /= L[3];
        int c2 = (int)(t % L[2]); t /= L[2];
        int c1 = (int)(t % L[1]); t /= L[1];
        int c0 = (int)t;
        if (((c0 + c1 + c2 + c3) & 1) == parity) memset(psi + 2 * s * ncomp, 0, sizeof(double) * 2 * ncomp);
    }
}

/* average (1/3) Re tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+ over x and mu<nu;
 * the reference's known answer for the Bridge++ 4^3x8 configuration is
 * 1 - CalculatePlaqutteEnergy(1/3)/(6V) = 0.625129946974942
 * (Code/CLGTest/Tests/TestConfigurationFileIO.cpp:12-38). */
double clgo_plaquette(const int L[4], const double* U) {
    const long V = volume(L);
    double total = 0;
#pragma omp parallel for schedule(static) reduction(+ : total)
    for (long s = 0; s < V; ++s) {
        long t = s;
        int c[4];
        c[3] = (int)(t % L[3]); t /= L[3];
        c[2] = (int)(t % L[2]); t /= L[2];
        c[1] = (int)(t % L[1]); t /= L[1];
        c[0] = (int)t;
        for (int mu = 0; mu < 4; ++mu)
            for (int nu = mu + 1; nu < 4; ++nu) {
                int a[4] = {c[0], c[1], c[2], c[3]}, b[4] = {c[0], c[1], c[2], c[3]};
                a[mu] = (a[mu] + 1) % L[mu];
                b[nu] = (b[nu] + 1) % L[nu];
                const long sa = (((long)a[0] * L[1] + a[1]) * L[2] + a[2]) * L[3] + a[3];
                const long sb = (((long)b[0] * L[1] + b[1]) * L[2] + b[2]) * L[3] + b[3];
                cplx u1[9], u2[9], u3[9], u4[9];
                load(U, s * 4 + mu, u1);
                load(U, sa * 4 + nu, u2);
                load(U, sb * 4 + mu, u3);
                load(U, s * 4 + nu, u4);
                /* tr(u1 u2 u3^+ u4^+) */
                cplx p[9], q[9];
                for (int r = 0; r < 3; ++r)
                    for (int cc = 0; cc < 3; ++cc)
                        p[3 * r + cc] = u1[3 * r] * u2[cc] + u1[3 * r + 1] * u2[3 + cc] + u1[3 * r + 2] * u2[6 + cc];
                /* q = u4 u3 ; tr(p q^+) = sum_ij p_ij conj(q_ij) */
                for (int r = 0; r < 3; ++r)
                    for (int cc = 0; cc < 3; ++cc)
                        q[3 * r + cc] = u4[3 * r] * u3[cc] + u4[3 * r + 1] * u3[3 + cc] + u4[3 * r + 2] * u3[6 + cc];
                double tr = 0;
                for (int k = 0; k < 9; ++k) tr += creal(p[k] * conj(q[k]));
                total += tr / 3.0;
            }
    }
    return total / (6.0 * (double)V);
}

double clgo_unitarity_deviation(long nlinks, const double* U) {
    double worst = 0;
    for (long l = 0; l < nlinks; ++l) {
        cplx m[9];
        load(U, l, m);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                cplx d = 0;
                for (int k = 0; k < 3; ++k) d += m[3 * r + k] * conj(m[3 * c + k]);
                const double e = cabs(d - (r == c ? 1.0 : 0.0));
                if (e > worst) worst = e;
            }
        const cplx det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                         m[2] * (m[3] * m[7] - m[4] * m[6]);
        const double e = cabs(det - 1.0);
        if (e > worst) worst = e;
    }
    return worst;
}

/* Bridge++ order: site = x + y Lx + z Lx Ly + t Lx Ly Lz, link = site*4 + mu, 18 reals
 * row-major (_kernelSetConfigurationSU3, CFieldGaugeSU3.cu:568-592). */
void clgo_bridgepp_to_clg(const int L[4], const double* bridge, double* U) {
    for (int x = 0; x < L[0]; ++x)
        for (int y = 0; y < L[1]; ++y)
            for (int z = 0; z < L[2]; ++z)
                for (int t = 0; t < L[3]; ++t) {
                    const long s = (((long)x * L[1] + y) * L[2] + z) * L[3] + t;
                    const long bs = x + (long)y * L[0] + (long)z * L[0] * L[1] + (long)t * L[0] * L[1] * L[2];
                    for (int mu = 0; mu < 4; ++mu)
                        memcpy(U + 18 * (s * 4 + mu), bridge + 18 * (bs * 4 + mu), sizeof(double) * 18);
                }
}
