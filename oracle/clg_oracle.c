/*
 * clg_oracle.c -- FP64 CPU restatement of CLGLib's Wilson / staggered Dirac
 * operators and the Krylov solvers that apply them.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline).  The
 * product library never links this file.  Reference paths below are relative
 * to the CudaLatticeGauge tree (Code/CLGLib/...).
 */
#include "clg_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex cplx;

/* ============================================================== geometry */

static inline long lat_volume(const int L[4]) { return (long)L[0] * L[1] * L[2] * L[3]; }

/* Data/CCommonData.h:274-277: s = ((x*Ly + y)*Lz + z)*Lt + t */
static inline long site_of(const int L[4], const int c[4]) {
    return (((long)c[0] * L[1] + c[1]) * L[2] + c[2]) * L[3] + c[3];
}
static inline void coords_of(const int L[4], long s, int c[4]) {
    c[3] = (int)(s % L[3]); s /= L[3];
    c[2] = (int)(s % L[2]); s /= L[2];
    c[1] = (int)(s % L[1]); s /= L[1];
    c[0] = (int)s;
}
/* neighbour x +/- mu with the torus wrap; *sign receives the boundary sign
 * (CBoundaryConditionTorusSquare.cu:18-64 multiplies bc[mu] per wrap). */
static inline long neighbour(const int L[4], const int bc[4], const int c[4], int mu, int fwd, int* sign) {
    int d[4] = {c[0], c[1], c[2], c[3]};
    int s = 1;
    if (fwd) {
        d[mu] += 1;
        if (d[mu] >= L[mu]) { d[mu] -= L[mu]; if (bc) s = bc[mu]; }
    } else {
        d[mu] -= 1;
        if (d[mu] < 0) { d[mu] += L[mu]; if (bc) s = bc[mu]; }
    }
    if (sign) *sign = s;
    return site_of(L, d);
}
static inline int parity_of(const int c[4]) { return (c[0] + c[1] + c[2] + c[3]) & 1; }

/* ============================================================== SU(3) helpers */

static inline void su3_load(const double* U, long link, cplx m[9]) {
    const double* p = U + 18 * link;
    for (int k = 0; k < 9; ++k) m[k] = p[2 * k] + I * p[2 * k + 1];
}
static inline void su3_store(double* U, long link, const cplx m[9]) {
    double* p = U + 18 * link;
    for (int k = 0; k < 9; ++k) { p[2 * k] = creal(m[k]); p[2 * k + 1] = cimag(m[k]); }
}
/* SU3.h:895-911 Dagger */
static inline void su3_dagger(const cplx a[9], cplx d[9]) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) d[3 * r + c] = conj(a[3 * c + r]);
}
static inline void su3_mul(const cplx a[9], const cplx b[9], cplx o[9]) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            o[3 * r + c] = a[3 * r] * b[c] + a[3 * r + 1] * b[3 + c] + a[3 * r + 2] * b[6 + c];
}
/* SU3.h:771-778 MulVector */
static inline void su3_mulvec(const cplx m[9], const cplx v[3], cplx o[3]) {
    o[0] = m[0] * v[0] + m[1] * v[1] + m[2] * v[2];
    o[1] = m[3] * v[0] + m[4] * v[1] + m[5] * v[2];
    o[2] = m[6] * v[0] + m[7] * v[1] + m[8] * v[2];
}

/* ============================================================== gamma matrices
 * Chiral set, Tools/Math/GammaMatrix.h:447-478: row r of gamma has a single
 * non-zero at column perm[r] with value i^z4[r].  MulWilsonC
 * (GammaMatrix.h:237-250): ret.d[r] = i^z4[r] * v.d[perm[r]].
 * Index 0..3 = GAMMA1..GAMMA4, 4 = GAMMA5. */
static const int g_perm[5][4] = {{3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1}, {2, 3, 0, 1}, {0, 1, 2, 3}};
static const int g_z4[5][4]   = {{3, 3, 1, 1}, {2, 0, 0, 2}, {3, 1, 1, 3}, {0, 0, 0, 0}, {0, 0, 2, 2}};

static inline cplx z4(int b) {
    switch (b & 3) {
        case 0: return 1.0;
        case 1: return I;
        case 2: return -1.0;
        default: return -I;
    }
}
/* spinor as 12 complex, index s*3+c */
static inline void gamma_mul(int g, const cplx in[12], cplx out[12]) {
    for (int r = 0; r < 4; ++r) {
        const cplx ph = z4(g_z4[g][r]);
        const int p = g_perm[g][r];
        for (int c = 0; c < 3; ++c) out[3 * r + c] = ph * in[3 * p + c];
    }
}

static inline void spinor_load(const double* f, long site, cplx v[12]) {
    const double* p = f + 24 * site;
    for (int k = 0; k < 12; ++k) v[k] = p[2 * k] + I * p[2 * k + 1];
}
static inline void spinor_store(double* f, long site, const cplx v[12]) {
    double* p = f + 24 * site;
    for (int k = 0; k < 12; ++k) { p[2 * k] = creal(v[k]); p[2 * k + 1] = cimag(v[k]); }
}
static inline void su3_mulwilson(const cplx m[9], const cplx in[12], cplx out[12]) {
    for (int s = 0; s < 4; ++s) su3_mulvec(m, in + 3 * s, out + 3 * s);
}

/* ============================================================== Wilson D
 * _kernelDFermionWilsonSquareSU3 (CFieldFermionWilsonSquareSU3.cu:32-163):
 *   out(x) = c * [ psi(x) - kappa sum_mu ( (1 - g_mu) U_mu(x) psi(x+mu) s_+
 *                                         + (1 + g_mu) U_mu(x-mu)^+ psi(x-mu) s_- ) ]
 * with s_+/- the boundary sign of the hop; dagger = g5 D g5 applied literally
 * (g5 on every gathered spinor and on the result, :53-56, :102-106, :149-152).
 * Coefficients as in DS (:909-933): EOCT_Minus becomes real -1.
 */
void clgo_wilson_D(const clgo_lat* lat, const double* U, double kappa, int dagger,
                   int coeff_type, double cre, double cim, const double* in, double* out) {
    const long V = lat_volume(lat->L);
    cplx coeff = 1.0;
    int apply_coeff = 0;
    if (coeff_type == CLGO_EOCT_MINUS) { coeff = -1.0; apply_coeff = 1; }
    else if (coeff_type == CLGO_EOCT_REAL) { coeff = cre; apply_coeff = 1; }
    else if (coeff_type == CLGO_EOCT_COMPLEX) { coeff = cre + I * cim; apply_coeff = 1; }

#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) {
        int c[4];
        coords_of(lat->L, s, c);
        cplx result[12] = {0};
        cplx self[12], tmp[12];
        spinor_load(in, s, self);
        if (dagger) { gamma_mul(4, self, tmp); memcpy(self, tmp, sizeof(self)); }
        for (int mu = 0; mu < 4; ++mu) {
            int sp, sm;
            const long xp = neighbour(lat->L, lat->bc, c, mu, 1, &sp);
            const long xm = neighbour(lat->L, lat->bc, c, mu, 0, &sm);
            cplx uf[9], ub0[9], ub[9];
            su3_load(U, s * 4 + mu, uf);
            su3_load(U, xm * 4 + mu, ub0);
            su3_dagger(ub0, ub);
            cplx pf[12], pb[12];
            spinor_load(in, xp, pf);
            spinor_load(in, xm, pb);
            if (dagger) {
                gamma_mul(4, pf, tmp); memcpy(pf, tmp, sizeof(pf));
                gamma_mul(4, pb, tmp); memcpy(pb, tmp, sizeof(pb));
            }
            cplx uphi[12], guphi[12];
            su3_mulwilson(uf, pf, uphi);
            gamma_mul(mu, uphi, guphi);
            for (int k = 0; k < 12; ++k) {
                if (sp < 0) { result[k] -= uphi[k]; result[k] += guphi[k]; }
                else        { result[k] += uphi[k]; result[k] -= guphi[k]; }
            }
            su3_mulwilson(ub, pb, uphi);
            gamma_mul(mu, uphi, guphi);
            for (int k = 0; k < 12; ++k) {
                if (sm < 0) { result[k] -= uphi[k]; result[k] -= guphi[k]; }
                else        { result[k] += uphi[k]; result[k] += guphi[k]; }
            }
        }
        cplx o[12];
        for (int k = 0; k < 12; ++k) o[k] = self[k] - kappa * result[k];
        if (dagger) { gamma_mul(4, o, tmp); memcpy(o, tmp, sizeof(o)); }
        if (apply_coeff) for (int k = 0; k < 12; ++k) o[k] *= coeff;
        spinor_store(out, s, o);
    }
}

/* Hopping term H restricted to output sites of one parity (the other parity of
 * `out` is set to zero).  D = 1 - kappa H, D^+ = 1 - kappa H^+ with
 * H^+ = g5 H g5, i.e. the projectors (1 -/+ g_mu) swap.  Even-odd split per
 * Docs/SparseLinearAlgebra/evenodd.tex:11-16 (D_ee = D_oo = 1 for Wilson). */
void clgo_wilson_hop(const clgo_lat* lat, const double* U, int dagger, int out_parity,
                     const double* in, double* out) {
    const long V = lat_volume(lat->L);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) {
        int c[4];
        coords_of(lat->L, s, c);
        cplx result[12] = {0};
        if (parity_of(c) == out_parity) {
            for (int mu = 0; mu < 4; ++mu) {
                int sp, sm;
                const long xp = neighbour(lat->L, lat->bc, c, mu, 1, &sp);
                const long xm = neighbour(lat->L, lat->bc, c, mu, 0, &sm);
                cplx uf[9], ub0[9], ub[9];
                su3_load(U, s * 4 + mu, uf);
                su3_load(U, xm * 4 + mu, ub0);
                su3_dagger(ub0, ub);
                cplx pf[12], pb[12], uphi[12], guphi[12];
                spinor_load(in, xp, pf);
                spinor_load(in, xm, pb);
                const double gsf = dagger ? 1.0 : -1.0; /* (1 - g) forward for D, (1 + g) for D^+ */
                su3_mulwilson(uf, pf, uphi);
                gamma_mul(mu, uphi, guphi);
                for (int k = 0; k < 12; ++k) result[k] += sp * (uphi[k] + gsf * guphi[k]);
                su3_mulwilson(ub, pb, uphi);
                gamma_mul(mu, uphi, guphi);
                for (int k = 0; k < 12; ++k) result[k] += sm * (uphi[k] - gsf * guphi[k]);
            }
        }
        spinor_store(out, s, result);
    }
}

/* M_ee = 1 - kappa^2 H_eo H_oe (evenodd.tex:11-16 with D_eo = -kappa H_eo).
 * Input/output are full-lattice arrays whose odd sites are ignored / zeroed. */
void clgo_wilson_mee(const clgo_lat* lat, const double* U, double kappa, int dagger,
                     const double* in, double* out, double* tmp) {
    const long V = lat_volume(lat->L);
    clgo_wilson_hop(lat, U, dagger, 1, in, tmp);
    clgo_wilson_hop(lat, U, dagger, 0, tmp, out);
    const double k2 = kappa * kappa;
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) {
        int c[4];
        coords_of(lat->L, s, c);
        const int even = parity_of(c) == 0;
        for (int k = 0; k < 24; ++k)
            out[24 * s + k] = even ? in[24 * s + k] - k2 * out[24 * s + k] : 0.0;
    }
}

/* ============================================================== Wilson fermion force
 * _kernelDWilsonForceSU3 (CFieldFermionWilsonSquareSU3.cu:170-231), launched by
 * DerivateDOperator (:260-275) from CalculateForceS (:1016-1100) with
 * X = (D D^+)^-1 phi (pInverseDDdagger) and Y = D^+ X (pInverseD):
 *   mid  = C(X(x), (1 - g_mu) Y(x+mu)) + C((1 + g_mu) Y(x), X(x+mu)),
 *          C(l, r) = sum_s r_s l_s^+   (makeSU3Contract, SU3.h:395-500)
 *   F_mu(x) += s_+ kappa Ta(U_mu(x) mid)
 * Ta: traceless anti-hermitian part (SU3.h:953-980); s_+ the boundary sign of
 * the hop to x+mu (NeedToOpposite).  F is added to, in the link layout of U. */
static inline void su3_ta(cplx m[9]) {
    for (int r = 0; r < 3; ++r)
        for (int c = r + 1; c < 3; ++c) {
            const cplx n = 0.5 * (m[3 * r + c] - conj(m[3 * c + r]));
            m[3 * r + c] = n;
            m[3 * c + r] = -conj(n);
        }
    const double tr = (cimag(m[0]) + cimag(m[4]) + cimag(m[8])) / 3.0;
    for (int d = 0; d < 3; ++d) m[4 * d] = I * (cimag(m[4 * d]) - tr);
}

void clgo_wilson_force(const clgo_lat* lat, const double* U, double kappa, const double* X, const double* Y,
                       double* F) {
    const long V = lat_volume(lat->L);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) {
        int c[4];
        coords_of(lat->L, s, c);
        cplx xl[12], xr[12];
        spinor_load(X, s, xl);
        spinor_load(Y, s, xr);
        for (int mu = 0; mu < 4; ++mu) {
            int sg = 1;
            const long sp = neighbour(lat->L, lat->bc, c, mu, 1, &sg);
            cplx xpl[12], xpr[12], g[12], r1[12], r2[12];
            spinor_load(X, sp, xpl);
            spinor_load(Y, sp, xpr);
            gamma_mul(mu, xpr, g);
            for (int k = 0; k < 12; ++k) r1[k] = xpr[k] - g[k];
            gamma_mul(mu, xr, g);
            for (int k = 0; k < 12; ++k) r2[k] = xr[k] + g[k];
            cplx mid[9];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    cplx v = 0;
                    for (int sp4 = 0; sp4 < 4; ++sp4)
                        v += conj(xl[3 * sp4 + b]) * r1[3 * sp4 + a] + conj(r2[3 * sp4 + b]) * xpl[3 * sp4 + a];
                    mid[3 * a + b] = v;
                }
            cplx u[9], m[9], f[9];
            su3_load(U, 4 * s + mu, u);
            su3_mul(u, mid, m);
            su3_ta(m);
            su3_load(F, 4 * s + mu, f);
            for (int k = 0; k < 9; ++k) f[k] += (double)sg * kappa * m[k];
            su3_store(F, 4 * s + mu, f);
        }
    }
}

/* ============================================================== staggered D
 * _kernelDFermionKS (CFieldFermionKSSU3.cu:33-117):
 *   out(x) = c * [ 2am chi(x) +/- sum_mu eta_mu(x) ( s_+ U_mu(x) chi(x+mu) - s_- U_mu(x-mu)^+ chi(x-mu) ) ]
 * "+" for D, "-" for D^+ (:100-107).  eta_mu(x) = (-1)^(x_0 + ... + x_{mu-1})
 * (SSmallInt4::EtaOdd, Data/CCommonData.h:228-236; table bits CIndexSquare.cu:255-265). */
static inline double eta_of(const int c[4], int mu) {
    int s = 0;
    for (int k = 0; k < mu; ++k) s += c[k];
    return (s & 1) ? -1.0 : 1.0;
}

static void ks_hop_site(const clgo_lat* lat, const double* U, const double* in, long s, const int c[4], cplx res[3]) {
    res[0] = res[1] = res[2] = 0;
    for (int mu = 0; mu < 4; ++mu) {
        int sp, sm;
        const long xp = neighbour(lat->L, lat->bc, c, mu, 1, &sp);
        const long xm = neighbour(lat->L, lat->bc, c, mu, 0, &sm);
        cplx uf[9], ub0[9], ub[9], vf[3], vb[3], a[3], b[3];
        su3_load(U, s * 4 + mu, uf);
        su3_load(U, xm * 4 + mu, ub0);
        su3_dagger(ub0, ub);
        for (int k = 0; k < 3; ++k) {
            vf[k] = in[6 * xp + 2 * k] + I * in[6 * xp + 2 * k + 1];
            vb[k] = in[6 * xm + 2 * k] + I * in[6 * xm + 2 * k + 1];
        }
        su3_mulvec(uf, vf, a);
        su3_mulvec(ub, vb, b);
        const double eta = eta_of(c, mu);
        for (int k = 0; k < 3; ++k) res[k] += eta * (sp * a[k] - sm * b[k]);
    }
}

void clgo_ks_D(const clgo_lat* lat, const double* U, double mass2am, int dagger,
               int coeff_type, double cre, double cim, const double* in, double* out) {
    const long V = lat_volume(lat->L);
    cplx coeff = 1.0;
    int apply_coeff = 0;
    if (coeff_type == CLGO_EOCT_MINUS) { coeff = -1.0; apply_coeff = 1; }
    else if (coeff_type == CLGO_EOCT_REAL) { coeff = cre; apply_coeff = 1; }
    else if (coeff_type == CLGO_EOCT_COMPLEX) { coeff = cre + I * cim; apply_coeff = 1; }
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) {
        int c[4];
        coords_of(lat->L, s, c);
        cplx h[3];
        ks_hop_site(lat, U, in, s, c, h);
        for (int k = 0; k < 3; ++k) {
            cplx self = in[6 * s + 2 * k] + I * in[6 * s + 2 * k + 1];
            cplx o = mass2am * self + (dagger ? -h[k] : h[k]);
            if (apply_coeff) o *= coeff;
            out[6 * s + 2 * k] = creal(o);
            out[6 * s + 2 * k + 1] = cimag(o);
        }
    }
}

void clgo_ks_hop(const clgo_lat* lat, const double* U, int out_parity, const double* in, double* out) {
    const long V = lat_volume(lat->L);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) {
        int c[4];
        coords_of(lat->L, s, c);
        cplx h[3] = {0, 0, 0};
        if (parity_of(c) == out_parity) ks_hop_site(lat, U, in, s, c, h);
        for (int k = 0; k < 3; ++k) { out[6 * s + 2 * k] = creal(h[k]); out[6 * s + 2 * k + 1] = cimag(h[k]); }
    }
}

/* (D D^+)_ee = (2am)^2 - H_eo H_oe : D = 2am + H with H anti-Hermitian
 * (comment at CFieldFermionKSSU3.cu:25-31), so D D^+ = (2am)^2 - H^2. */
void clgo_ks_dddag_ee(const clgo_lat* lat, const double* U, double mass2am,
                      const double* in, double* out, double* tmp) {
    const long V = lat_volume(lat->L);
    clgo_ks_hop(lat, U, 1, in, tmp);
    clgo_ks_hop(lat, U, 0, tmp, out);
    const double m2 = mass2am * mass2am;
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) {
        int c[4];
        coords_of(lat->L, s, c);
        const int even = parity_of(c) == 0;
        for (int k = 0; k < 6; ++k) out[6 * s + k] = even ? m2 * in[6 * s + k] - out[6 * s + k] : 0.0;
    }
}

/* ============================================================== staggered rational force
 * _kernelDFermionKSForce (Staggered/CFieldFermionKSSU3.cu:216-262), launched by
 * DerivateD0 (:316-331) from CalculateForceS (:412-500): with the multi-shift
 * solutions phi_i = (D D^+ + b_i)^-1 phi and phi_id = D0 phi_i (the massless D),
 *   F_mu(x) -= Ta( s_+ eta_mu(x) a_i [ U_mu(x) phi_i(x+mu) phi_id(x)^+
 *                                     + phi_i(x) (U_mu(x) phi_id(x+mu))^+ ] )
 * summed over i (makeSU3ContractV(l, r) = r l^+, SU3.h:505-519).  phi_i and
 * phi_id hold n fields of V*3 complex one after another. */
void clgo_ks_force(const clgo_lat* lat, const double* U, int n, const double* phi_i, const double* phi_id,
                   const double* a, double* F) {
    const long V = lat_volume(lat->L);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; ++s) {
        int c[4];
        coords_of(lat->L, s, c);
        for (int mu = 0; mu < 4; ++mu) {
            int sg = 1;
            const long sp = neighbour(lat->L, lat->bc, c, mu, 1, &sg);
            cplx u[9], f[9], term[9];
            su3_load(U, 4 * s + mu, u);
            su3_load(F, 4 * s + mu, f);
            const double w0 = eta_of(c, mu) * (double)sg;
            for (int i = 0; i < n; ++i) {
                const double* pi = phi_i + (long)i * 6 * V;
                const double* pd = phi_id + (long)i * 6 * V;
                cplx vi_x[3], vd_x[3], vi_p[3], vd_p[3], t1[3], t2[3];
                for (int k = 0; k < 3; ++k) {
                    vi_x[k] = pi[6 * s + 2 * k] + I * pi[6 * s + 2 * k + 1];
                    vd_x[k] = pd[6 * s + 2 * k] + I * pd[6 * s + 2 * k + 1];
                    vi_p[k] = pi[6 * sp + 2 * k] + I * pi[6 * sp + 2 * k + 1];
                    vd_p[k] = pd[6 * sp + 2 * k] + I * pd[6 * sp + 2 * k + 1];
                }
                su3_mulvec(u, vi_p, t1);
                su3_mulvec(u, vd_p, t2);
                for (int r = 0; r < 3; ++r)
                    for (int q = 0; q < 3; ++q)
                        term[3 * r + q] = t1[r] * conj(vd_x[q]) + vi_x[r] * conj(t2[q]);
                const double w = w0 * a[i];
                for (int k = 0; k < 9; ++k) term[k] *= w;
                su3_ta(term);
                for (int k = 0; k < 9; ++k) f[k] -= term[k];
            }
            su3_store(F, 4 * s + mu, f);
        }
    }
}

/* ============================================================== generic op */
long clgo_op_len(const clgo_op* op) {
    const long V = lat_volume(op->lat.L);
    return (op->kind >= CLGO_OP_KS_D) ? 3 * V : 12 * V;
}

void clgo_apply(const clgo_op* op, const double* in, double* out) {
    const clgo_lat* lat = &op->lat;
    switch (op->kind) {
        case CLGO_OP_WILSON_D:
            clgo_wilson_D(lat, op->U, op->param, 0, 0, 0, 0, in, out); break;
        case CLGO_OP_WILSON_DDAG:
            clgo_wilson_D(lat, op->U, op->param, 1, 0, 0, 0, in, out); break;
        case CLGO_OP_WILSON_DDDAG: /* DDdaggerS: D(D^+ x) (CFieldFermionWilsonSquareSU3.cu:962-987) */
            clgo_wilson_D(lat, op->U, op->param, 1, 0, 0, 0, in, op->tmp);
            clgo_wilson_D(lat, op->U, op->param, 0, 0, 0, 0, op->tmp, out); break;
        case CLGO_OP_WILSON_DD:
            clgo_wilson_D(lat, op->U, op->param, 0, 0, 0, 0, in, op->tmp);
            clgo_wilson_D(lat, op->U, op->param, 0, 0, 0, 0, op->tmp, out); break;
        case CLGO_OP_WILSON_MEE:
            clgo_wilson_mee(lat, op->U, op->param, 0, in, out, op->tmp); break;
        case CLGO_OP_WILSON_MEE_DAG:
            clgo_wilson_mee(lat, op->U, op->param, 1, in, out, op->tmp); break;
        case CLGO_OP_WILSON_MEE_MEEDAG:
            clgo_wilson_mee(lat, op->U, op->param, 1, in, op->tmp2, op->tmp);
            clgo_wilson_mee(lat, op->U, op->param, 0, op->tmp2, out, op->tmp); break;
        case CLGO_OP_KS_D:
            clgo_ks_D(lat, op->U, op->param, 0, 0, 0, 0, in, out); break;
        case CLGO_OP_KS_DDAG:
            clgo_ks_D(lat, op->U, op->param, 1, 0, 0, 0, in, out); break;
        case CLGO_OP_KS_DDDAG: /* DDdaggerS (CFieldFermionKSSU3.cu:1550-1575) */
            clgo_ks_D(lat, op->U, op->param, 1, 0, 0, 0, in, op->tmp);
            clgo_ks_D(lat, op->U, op->param, 0, 0, 0, 0, op->tmp, out); break;
        case CLGO_OP_KS_DDDAG_EE:
            clgo_ks_dddag_ee(lat, op->U, op->param, in, out, op->tmp); break;
        default: break;
    }
}

/* ============================================================== BLAS
 * Dot = sum conj(a) b (CFieldFermionWilsonSquareSU3.cu:394-411, 832-844),
 * accumulated here in long double over fixed chunks so the result does not
 * depend on the thread count. */
#define CLGO_CHUNKS 256
void clgo_dot(long n, const double* a, const double* b, double* re_im) {
    long double pr[CLGO_CHUNKS], pi[CLGO_CHUNKS];
#pragma omp parallel for schedule(static)
    for (int ch = 0; ch < CLGO_CHUNKS; ++ch) {
        const long lo = n * ch / CLGO_CHUNKS, hi = n * (ch + 1) / CLGO_CHUNKS;
        long double sr = 0, si = 0;
        for (long k = lo; k < hi; ++k) {
            const double ar = a[2 * k], ai = a[2 * k + 1], br = b[2 * k], bi = b[2 * k + 1];
            sr += (long double)ar * br + (long double)ai * bi;
            si += (long double)ar * bi - (long double)ai * br;
        }
        pr[ch] = sr; pi[ch] = si;
    }
    long double sr = 0, si = 0;
    for (int ch = 0; ch < CLGO_CHUNKS; ++ch) { sr += pr[ch]; si += pi[ch]; }
    re_im[0] = (double)sr; re_im[1] = (double)si;
}
double clgo_norm2(long n, const double* a) { double d[2]; clgo_dot(n, a, a, d); return d[0]; }

void clgo_axpy(long n, double are, double aim, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (long k = 0; k < n; ++k) {
        const double xr = x[2 * k], xi = x[2 * k + 1];
        y[2 * k] += are * xr - aim * xi;
        y[2 * k + 1] += are * xi + aim * xr;
    }
}
static inline cplx cdot(long n, const double* a, const double* b) { double d[2]; clgo_dot(n, a, b, d); return d[0] + I * d[1]; }
static inline void caxpy(long n, cplx a, const double* x, double* y) { clgo_axpy(n, creal(a), cimag(a), x, y); }
static void cscale(long n, cplx a, double* y) {
#pragma omp parallel for schedule(static)
    for (long k = 0; k < n; ++k) {
        const double yr = y[2 * k], yi = y[2 * k + 1];
        y[2 * k] = creal(a) * yr - cimag(a) * yi;
        y[2 * k + 1] = creal(a) * yi + cimag(a) * yr;
    }
}
static void vcopy(long n, const double* x, double* y) { memcpy(y, x, sizeof(double) * 2 * n); }
static double* valloc(long n) { return (double*)calloc((size_t)(2 * n), sizeof(double)); }

double clgo_true_residual(const clgo_op* op, const double* b, const double* x, double shift_re, double shift_im) {
    const long n = clgo_op_len(op);
    double* r = valloc(n);
    clgo_apply(op, x, r);
    if (shift_re != 0.0 || shift_im != 0.0) caxpy(n, shift_re + I * shift_im, x, r);
#pragma omp parallel for schedule(static)
    for (long k = 0; k < 2 * n; ++k) r[k] = b[k] - r[k];
    const double rn = clgo_norm2(n, r), bn = clgo_norm2(n, b);
    free(r);
    return bn > 0 ? sqrt(rn / bn) : sqrt(rn);
}

/* ============================================================== GMRES(k)
 * CSLASolverGMRES::Solve (SparseLinearAlgebra/CSolverGMRES.cpp:111-260):
 * restarted GMRES, modified Gram-Schmidt Arnoldi of fixed length MaxDim,
 * Givens rotations RotateH (:262-327), back substitution SolveY (:329-358);
 * stop when |g_m|^2 < Accuracy * fBLength (fBLength = |b|^2 unless
 * AbsoluteAccuracy, :128-131, :232). */
int clgo_gmres(const clgo_op* op, const double* b, double* x, const double* x0,
               int maxdim, int restart, double accuracy, int absolute, clgo_info* info) {
    const long n = clgo_op_len(op);
    const int m = maxdim;
    double** v = (double**)malloc(sizeof(double*) * m);
    for (int i = 0; i < m; ++i) v[i] = valloc(n);
    double* X = valloc(n);
    double* W = valloc(n);
    cplx* h = (cplx*)calloc((size_t)(m + 1) * m, sizeof(cplx)); /* h[k*m + j] */
    cplx* g = (cplx*)calloc((size_t)(m + 1), sizeof(cplx));
    cplx* y = (cplx*)calloc((size_t)m, sizeof(cplx));
    const double blen = absolute ? 1.0 : clgo_norm2(n, b);
    vcopy(n, x0 ? x0 : b, X);
    double last = 0;
    int napply = 0, converged = 0, cycles = 0;
    for (int it = 0; it < restart; ++it) {
        ++cycles;
        clgo_apply(op, X, v[0]); ++napply;
#pragma omp parallel for schedule(static)
        for (long k = 0; k < 2 * n; ++k) v[0][k] = b[k] - v[0][k];
        const double beta = sqrt(clgo_norm2(n, v[0]));
        cscale(n, 1.0 / beta, v[0]);
        for (int j = 0; j < m; ++j) {
            clgo_apply(op, v[j], W); ++napply;
            for (int k = 0; k <= j; ++k) {
                const cplx d = cdot(n, v[k], W);
                h[k * m + j] = d;
                caxpy(n, -d, v[k], W);
            }
            const double wn = sqrt(clgo_norm2(n, W));
            h[(j + 1) * m + j] = wn;
            if (j < m - 1) { cscale(n, 1.0 / wn, W); vcopy(n, W, v[j + 1]); }
        }
        /* RotateH */
        g[0] = beta;
        for (int i = 0; i < m; ++i) {
            const cplx hii = h[i * m + i], hi1 = h[(i + 1) * m + i];
            const double den = 1.0 / sqrt(creal(hii * conj(hii)) + creal(hi1 * conj(hi1)));
            const cplx cs = hii * den, sn = hi1 * den;
            for (int j = i; j < m; ++j) {
                const cplx hij = h[i * m + j];
                h[i * m + j] = conj(cs) * hij + conj(sn) * h[(i + 1) * m + j];
                h[(i + 1) * m + j] = cs * h[(i + 1) * m + j] - sn * hij;
            }
            const cplx mg = -g[i];
            g[i] = conj(cs) * g[i];
            g[i + 1] = sn * mg;
        }
        last = creal(g[m] * conj(g[m]));
        /* SolveY */
        for (int i = m - 1; i >= 0; --i) {
            for (int j = i + 1; j < m; ++j) g[i] -= h[i * m + j] * y[j];
            y[i] = g[i] / h[i * m + i];
        }
        for (int j = 0; j < m; ++j) caxpy(n, y[j], v[j], X);
        if (last < accuracy * blen) { converged = 1; break; }
    }
    vcopy(n, X, x);
    if (info) {
        info->iterations = napply; info->restarts = cycles; info->converged = converged;
        info->last_deviation = last; info->true_rel_residual = clgo_true_residual(op, b, x, 0, 0);
    }
    for (int i = 0; i < m; ++i) free(v[i]);
    free(v); free(X); free(W); free(h); free(g); free(y);
    return converged;
}

/* ============================================================== BiCGStab
 * CSLASolverBiCGStab::Solve (SparseLinearAlgebra/CSolverBiCGstab.cpp:403-607):
 * r^ = conj(r0) (so rho is the unconjugated bilinear sum r0 r), restart after
 * MaxStep*DiviationStep steps, check |s|^2/|b|^2 < Accuracy every DiviationStep
 * and return x WITHOUT the final alpha p update (:525). */
int clgo_bicgstab(const clgo_op* op, const double* b, double* x, const double* x0,
                  int dev_step, int max_step, int restart, double accuracy, int absolute,
                  double small_rho, int std_omega, clgo_info* info) {
    const long n = clgo_op_len(op);
    double *X = valloc(n), *P = valloc(n), *Vv = valloc(n), *R = valloc(n), *Rh = valloc(n), *S = valloc(n), *T = valloc(n);
    const double blen = absolute ? 1.0 : clgo_norm2(n, b);   /* _cuCabsf(b.Dot(b)) (:425-431) */
    vcopy(n, x0 ? x0 : b, R);
    vcopy(n, x0 ? x0 : b, X);
    int napply = 0, converged = 0, cycles = 0;
    double last = 0;
    for (int i = 0; i < restart && !converged; ++i) {
        ++cycles;
        clgo_apply(op, R, T); ++napply;  /* R currently holds x */
#pragma omp parallel for schedule(static)
        for (long k = 0; k < 2 * n; ++k) R[k] = b[k] - T[k];
        vcopy(n, R, Rh);
#pragma omp parallel for schedule(static)
        for (long k = 0; k < n; ++k) Rh[2 * k + 1] = -Rh[2 * k + 1];
        vcopy(n, R, P);
        cplx rho = 0, alpha = 0, beta = 0, omega = 0;
        int broke = 0;
        for (int j = 0; j < max_step * dev_step; ++j) {
            if (j == 0) rho = cdot(n, Rh, R);
            /* last retry: _CLG_FLT_MIN of the FP64 build (Core/CLGFloat.h:115) */
            const double lim = (restart == i + 1) ? 2.2250738585072014e-308 : small_rho;
            if (creal(rho * conj(rho)) < lim) { broke = 1; ++i; break; }
            clgo_apply(op, P, Vv); ++napply;
            alpha = rho / cdot(n, Rh, Vv);
            vcopy(n, R, S);
            caxpy(n, -alpha, Vv, S);
            if ((j + 1) % dev_step == 0) {
                last = clgo_norm2(n, S) / blen;
                if (last < accuracy) { converged = 1; break; }
            }
            clgo_apply(op, S, T); ++napply;
            /* reference (:527-533): omega = pS->Dot(pT) / |t|^2 = sum conj(s) t / |t|^2;
             * std_omega selects the residual-minimising sum conj(t) s / |t|^2 */
            omega = (std_omega ? cdot(n, T, S) : cdot(n, S, T)) / clgo_norm2(n, T);
            vcopy(n, S, R);
            caxpy(n, -omega, T, R);
            beta = alpha / (omega * rho);
            rho = cdot(n, Rh, R);
            beta = beta * rho;
            caxpy(n, alpha, P, X);
            caxpy(n, omega, S, X);
            cscale(n, omega, Vv);
#pragma omp parallel for schedule(static)
            for (long k = 0; k < 2 * n; ++k) P[k] -= Vv[k];
            cscale(n, beta, P);
#pragma omp parallel for schedule(static)
            for (long k = 0; k < 2 * n; ++k) P[k] += R[k];
        }
        (void)broke;
        if (!converged) vcopy(n, X, R);
    }
    vcopy(n, X, x);
    if (info) {
        info->iterations = napply; info->restarts = cycles; info->converged = converged;
        info->last_deviation = last; info->true_rel_residual = clgo_true_residual(op, b, x, 0, 0);
    }
    free(X); free(P); free(Vv); free(R); free(Rh); free(S); free(T);
    return converged;
}

/* ============================================================== CG
 * Plain conjugate gradient for Hermitian positive-definite operators (used for
 * the staggered (D D^+)_ee system).  Stops on the recursive residual. */
int clgo_cg(const clgo_op* op, const double* b, double* x, double tol_rel, int maxiter, clgo_info* info) {
    const long n = clgo_op_len(op);
    double *r = valloc(n), *p = valloc(n), *q = valloc(n);
    memset(x, 0, sizeof(double) * 2 * n);
    vcopy(n, b, r); vcopy(n, b, p);
    const double bn = clgo_norm2(n, b);
    double rr = bn;
    int it = 0, conv = 0;
    for (; it < maxiter; ++it) {
        if (rr <= tol_rel * tol_rel * bn) { conv = 1; break; }
        clgo_apply(op, p, q);
        const double pq = creal(cdot(n, p, q));
        const double a = rr / pq;
        caxpy(n, a, p, x);
        caxpy(n, -a, q, r);
        const double rr2 = clgo_norm2(n, r);
        const double be = rr2 / rr;
        rr = rr2;
        cscale(n, be, p);
        caxpy(n, 1.0, r, p);
    }
    if (info) {
        info->iterations = it; info->restarts = 1; info->converged = conv;
        info->last_deviation = sqrt(rr / bn); info->true_rel_residual = clgo_true_residual(op, b, x, 0, 0);
    }
    free(r); free(p); free(q);
    return conv;
}

/* ============================================================== CG-M
 * Multi-shift CG (B. Jegerlehner, "Krylov space solvers for shifted linear
 * systems", hep-lat/9612014): solves (A + sigma_k) x_k = b for all k over the
 * Krylov space of the base system A (shift 0).  The reference has no CG-M;
 * its multi-shift family is CMultiShiftFOM / GMRES / BiCGStab
 * (SparseLinearAlgebra/CMultiShift*.cpp) with the interface of
 * CMultiShiftSolver.h:38-47.  x is nshift consecutive fields. */
int clgo_cgm(const clgo_op* op, const double* b, int nshift, const double* shifts, double* x,
             double tol_rel, int maxiter, clgo_info* info) {
    const long n = clgo_op_len(op);
    double *r = valloc(n), *p = valloc(n), *q = valloc(n);
    double* ps = valloc(n * nshift);
    double *zeta = calloc(nshift, sizeof(double)), *zeta_old = calloc(nshift, sizeof(double));
    double *alpha_s = calloc(nshift, sizeof(double)), *beta_s = calloc(nshift, sizeof(double));
    int* active = calloc(nshift, sizeof(int));
    memset(x, 0, sizeof(double) * 2 * n * nshift);
    vcopy(n, b, r); vcopy(n, b, p);
    for (int k = 0; k < nshift; ++k) { vcopy(n, b, ps + 2 * n * k); zeta[k] = zeta_old[k] = 1.0; active[k] = 1; }
    const double bn = clgo_norm2(n, b);
    double rr = bn, alpha_old = 1.0, beta = 0.0;
    int it = 0, conv = 0;
    for (; it < maxiter; ++it) {
        clgo_apply(op, p, q);
        const double pq = creal(cdot(n, p, q));
        const double alpha = rr / pq;
        caxpy(n, -alpha, q, r);
        const double rr2 = clgo_norm2(n, r);
        const double beta_new = rr2 / rr;
        int nact = 0;
        for (int k = 0; k < nshift; ++k) {
            if (!active[k]) continue;
            const double sg = shifts[k];
            /* zeta_{n+1} = zeta_n zeta_{n-1} a_{n-1} / (a_n b_{n-1}(zeta_{n-1}-zeta_n) + zeta_{n-1} a_{n-1}(1 + sigma a_n)) */
            const double zn = zeta[k], zo = zeta_old[k];
            const double den = alpha * beta * (zo - zn) + zo * alpha_old * (1.0 + sg * alpha);
            const double znew = zn * zo * alpha_old / den;
            const double as = alpha * znew / zn;
            caxpy(n, as, ps + 2 * n * k, x + 2 * n * k);
            const double bs = beta_new * (znew / zn) * (znew / zn);
            /* p_s = zeta_new r + beta_s p_s */
            double* pk = ps + 2 * n * k;
#pragma omp parallel for schedule(static)
            for (long j = 0; j < 2 * n; ++j) pk[j] = znew * r[j] + bs * pk[j];
            zeta_old[k] = zn; zeta[k] = znew; alpha_s[k] = as; beta_s[k] = bs;
            if (fabs(znew) * fabs(znew) * rr2 <= tol_rel * tol_rel * bn) active[k] = 0;
            else ++nact;
        }
        cscale(n, beta_new, p);
        caxpy(n, 1.0, r, p);
        alpha_old = alpha; beta = beta_new; rr = rr2;
        if (nact == 0 && rr <= tol_rel * tol_rel * bn) { conv = 1; ++it; break; }
        if (nact == 0) { conv = 1; ++it; break; }
    }
    if (info) {
        info->iterations = it; info->restarts = 1; info->converged = conv;
        double worst = 0;
        for (int k = 0; k < nshift; ++k) {
            const double t = clgo_true_residual(op, b, x + 2 * n * k, shifts[k], 0.0);
            if (t > worst) worst = t;
        }
        info->last_deviation = sqrt(rr / bn);
        info->true_rel_residual = worst;
    }
    free(r); free(p); free(q); free(ps); free(zeta); free(zeta_old); free(alpha_s); free(beta_s); free(active);
    return conv;
}

/* ============================================================== FOM-M
 * CMultiShiftFOM::Solve (SparseLinearAlgebra/CMultiShiftFOM.cpp:97-270):
 * a shared Arnoldi basis of length MaxDim on A; for each shift c_n solve the
 * FOM system (H_m + c_n) y = beta0_n e_1, x_n += V y, and the new residual
 * coefficient beta0_n = -y_{m-1} h_{m,m-1} on the shared restart vector
 * v_m.  Stop when max_n |beta0_n| < Accuracy * fBLength.  shifts_c holds
 * nshift complex (re,im) pairs; x is nshift consecutive fields. */
int clgo_fom_ms(const clgo_op* op, const double* b, int nshift, const double* shifts_c, double* x,
                int maxdim, int restart, double accuracy, int absolute, clgo_info* info) {
    const long n = clgo_op_len(op);
    const int m = maxdim;
    double** v = (double**)malloc(sizeof(double*) * m);
    for (int i = 0; i < m; ++i) v[i] = valloc(n);
    double *W = valloc(n), *R = valloc(n);
    cplx* h = (cplx*)calloc((size_t)(m + 1) * m, sizeof(cplx));
    cplx* hc = (cplx*)calloc((size_t)m * m, sizeof(cplx));
    cplx* y = (cplx*)calloc((size_t)m, sizeof(cplx));
    cplx* beta0 = (cplx*)calloc((size_t)nshift, sizeof(cplx));
    double* beta0len = (double*)calloc((size_t)nshift, sizeof(double));
    /* fBLength = pFieldB->GetLength() = |b|^2 (CMultiShiftFOM.cpp:118-121), compared with |beta_n| */
    const double blen = absolute ? 1.0 : clgo_norm2(n, b);
    memset(x, 0, sizeof(double) * 2 * n * nshift);
    int napply = 0, converged = 0, cycles = 0;
    double maxerr = 0;
    for (int it = 0; it < restart; ++it) {
        ++cycles;
        if (it == 0) vcopy(n, b, R);
        vcopy(n, R, v[0]);
        if (it == 0) {
            const double beta = sqrt(clgo_norm2(n, v[0]));
            for (int s = 0; s < nshift; ++s) { beta0[s] = beta; beta0len[s] = beta; }
            cscale(n, 1.0 / beta, v[0]);
        }
        for (int j = 0; j < m; ++j) {
            clgo_apply(op, v[j], W); ++napply;
            for (int k = 0; k <= j; ++k) {
                const cplx d = cdot(n, v[k], W);
                h[k * m + j] = d;
                caxpy(n, -d, v[k], W);
            }
            const double wn = sqrt(clgo_norm2(n, W));
            h[(j + 1) * m + j] = wn;
            cscale(n, 1.0 / wn, W);
            vcopy(n, W, (j < m - 1) ? v[j + 1] : R);
        }
        maxerr = 0;
        for (int s = 0; s < nshift; ++s) {
            if (beta0len[s] < accuracy * blen) continue;
            const cplx cs = shifts_c[2 * s] + I * shifts_c[2 * s + 1];
            for (int r = 0; r < m; ++r)
                for (int c = 0; c < m; ++c) hc[r * m + c] = h[r * m + c] + (r == c ? cs : 0.0);
            /* Gaussian elimination with partial pivoting on the m x m Hessenberg
             * (the reference uses Givens rotations + back substitution;
             * the solution is the same up to rounding) */
            cplx rhs[128];
            for (int r = 0; r < m; ++r) rhs[r] = (r == 0) ? beta0[s] : 0.0;
            for (int col = 0; col < m; ++col) {
                int piv = col;
                for (int r = col + 1; r < m; ++r) if (cabs(hc[r * m + col]) > cabs(hc[piv * m + col])) piv = r;
                if (piv != col) {
                    for (int c = 0; c < m; ++c) { cplx t = hc[col * m + c]; hc[col * m + c] = hc[piv * m + c]; hc[piv * m + c] = t; }
                    cplx t = rhs[col]; rhs[col] = rhs[piv]; rhs[piv] = t;
                }
                for (int r = col + 1; r < m; ++r) {
                    const cplx f = hc[r * m + col] / hc[col * m + col];
                    if (f == 0) continue;
                    for (int c = col; c < m; ++c) hc[r * m + c] -= f * hc[col * m + c];
                    rhs[r] -= f * rhs[col];
                }
            }
            for (int r = m - 1; r >= 0; --r) {
                cplx acc = rhs[r];
                for (int c = r + 1; c < m; ++c) acc -= hc[r * m + c] * y[c];
                y[r] = acc / hc[r * m + r];
            }
            beta0[s] = -y[m - 1] * creal(h[m * m + (m - 1)]);
            const double e = cabs(beta0[s]);
            beta0len[s] = e;
            if (e > maxerr) maxerr = e;
            for (int j = 0; j < m; ++j) caxpy(n, y[j], v[j], x + 2 * n * s);
        }
        if (maxerr < accuracy * blen) { converged = 1; break; }
        /* the restart vector R carries unit norm; each shift's residual is beta0[s] R */
        /* for the next cycle the shared basis starts from R and every shift's
         * right-hand side is beta0[s] e_1 */
        vcopy(n, R, R);
    }
    if (info) {
        info->iterations = napply; info->restarts = cycles; info->converged = converged;
        info->last_deviation = maxerr;
        double worst = 0;
        for (int s = 0; s < nshift; ++s) {
            const double t = clgo_true_residual(op, b, x + 2 * n * s, shifts_c[2 * s], shifts_c[2 * s + 1]);
            if (t > worst) worst = t;
        }
        info->true_rel_residual = worst;
    }
    for (int i = 0; i < m; ++i) free(v[i]);
    free(v); free(W); free(R); free(h); free(hc); free(y); free(beta0); free(beta0len);
    return converged;
}

/* ============================================================== multi-shift BiCGStab
 * CMultiShiftBiCGStab::Solve (SparseLinearAlgebra/CMultiShiftBiCGStab.cpp:73-437;
 * B. Jegerlehner, hep-lat/9612014): (A + c_n) x_n = b for every shift over the
 * BiCGStab recurrences of A, with the shadow residual w0 = conj(b) (the
 * reference's Dagger of b).  Every `dev_step` iterations the residual estimates
 * |s| and |s_n| are compared with accuracy * |b| (|b| = 1 when absolute).
 * x holds nshift solutions of length n; shifts_c interleaved complex. */
int clgo_bicgstab_ms(const clgo_op* op, const double* b, int nshift, const double* shifts_c, double* x,
                     int dev_step, int max_step, double accuracy, int absolute, clgo_info* info) {
    const long n = clgo_op_len(op);
    double *R = valloc(n), *W = valloc(n), *W0 = valloc(n), *S = valloc(n), *SA = valloc(n), *WA = valloc(n);
    double** Ss = (double**)malloc(sizeof(double*) * nshift);
    cplx *betas = (cplx*)malloc(sizeof(cplx) * nshift), *zeta = (cplx*)malloc(sizeof(cplx) * nshift),
         *zetaold = (cplx*)malloc(sizeof(cplx) * nshift), *rho = (cplx*)malloc(sizeof(cplx) * nshift),
         *alphas = (cplx*)malloc(sizeof(cplx) * nshift);
    double* sl = (double*)malloc(sizeof(double) * nshift);
    memset(x, 0, sizeof(double) * 2 * n * nshift);
    for (int s = 0; s < nshift; ++s) {
        Ss[s] = valloc(n);
        vcopy(n, b, Ss[s]);
        betas[s] = 1; zeta[s] = 1; zetaold[s] = 1; rho[s] = 1; alphas[s] = 0; sl[s] = 1.0;
    }
    const double blen = absolute ? 1.0 : sqrt(clgo_norm2(n, b));
    vcopy(n, b, R); vcopy(n, b, W); vcopy(n, b, S); vcopy(n, b, SA);
    vcopy(n, b, W0);
    for (long k = 0; k < n; ++k) W0[2 * k + 1] = -W0[2 * k + 1];   /* pW->Dagger() */
    cplx delta = cdot(n, W0, R);
    double* T = valloc(n);
    clgo_apply(op, SA, T); vcopy(n, T, SA);
    int napply = 1;
    cplx phi = cdot(n, W0, SA) / delta;
    cplx beta = 0, alpha = 0;
    int done = 0, it = 0;
    double maxerr = 0;
    for (it = 0; it < max_step * dev_step; ++it) {
        const cplx newbeta = -1.0 / phi;
        for (int s = 0; s < nshift; ++s) {
            if (sl[s] < accuracy * blen) continue;
            const cplx c = shifts_c[2 * s] + I * shifts_c[2 * s + 1];
            if (it == 0) {
                zeta[s] = 1.0 / (1.0 - c * newbeta);
                betas[s] = newbeta * zeta[s];
            } else {
                const cplx znm1 = zetaold[s];
                zetaold[s] = zeta[s];
                const cplx zb = znm1 * beta;
                zeta[s] = (zetaold[s] * zb) / (alpha * (newbeta * (znm1 - zetaold[s])) + zb * (1.0 - c * newbeta));
                betas[s] = newbeta * zeta[s] / zetaold[s];
            }
        }
        beta = newbeta;
        vcopy(n, R, W);
        caxpy(n, beta, SA, W);
        clgo_apply(op, W, WA); ++napply;
        const cplx chi = cdot(n, WA, W) / clgo_norm2(n, WA);
        for (int s = 0; s < nshift; ++s) {
            if (sl[s] < accuracy * blen) continue;
            const cplx c = shifts_c[2 * s] + I * shifts_c[2 * s + 1];
            const cplx dinom = 1.0 + c * chi;
            const cplx chis = chi / dinom;
            const cplx chirho = chis * rho[s];
            const cplx crz = chirho * zeta[s];
            double* xs = x + 2 * n * s;
            caxpy(n, -betas[s], Ss[s], xs);
            caxpy(n, crz, W, xs);
            caxpy(n, -(crz / betas[s]), W, Ss[s]);
            caxpy(n, chirho * zetaold[s] / betas[s], R, Ss[s]);
            rho[s] = rho[s] / dinom;
        }
        vcopy(n, W, R);
        caxpy(n, -chi, WA, R);
        const cplx newdelta = cdot(n, W0, R);
        alpha = (beta * (-newdelta)) / (chi * delta);
        delta = newdelta;
        for (int s = 0; s < nshift; ++s) {
            if (sl[s] < accuracy * blen) continue;
            alphas[s] = (alpha * zeta[s] * betas[s]) / (zetaold[s] * beta);
            cscale(n, alphas[s], Ss[s]);
            caxpy(n, zeta[s] * rho[s], R, Ss[s]);
        }
        caxpy(n, -chi, SA, S);
        cscale(n, alpha, S);
        caxpy(n, 1.0, R, S);
        clgo_apply(op, S, SA); ++napply;
        phi = cdot(n, W0, SA) / delta;
        if ((it + 1) % dev_step == 0) {
            maxerr = sqrt(clgo_norm2(n, S));
            for (int s = 0; s < nshift; ++s) {
                if (sl[s] < accuracy * blen) continue;
                sl[s] = sqrt(clgo_norm2(n, Ss[s]));
                if (sl[s] > maxerr) maxerr = sl[s];
            }
            if (maxerr < accuracy * blen) { done = 1; break; }
        }
    }
    if (info) {
        info->iterations = napply; info->restarts = it; info->converged = done;
        info->last_deviation = maxerr;
        double worst = 0;
        for (int s = 0; s < nshift; ++s) {
            const double t = clgo_true_residual(op, b, x + 2 * n * s, shifts_c[2 * s], shifts_c[2 * s + 1]);
            if (t > worst) worst = t;
        }
        info->true_rel_residual = worst;
    }
    for (int s = 0; s < nshift; ++s) free(Ss[s]);
    free(Ss); free(betas); free(zeta); free(zetaold); free(rho); free(alphas); free(sl);
    free(R); free(W); free(W0); free(S); free(SA); free(WA); free(T);
    return done;
}

/* ============================================================== multi-shift GMRES
 * CMultiShiftGMRES::Solve (SparseLinearAlgebra/CMultiShiftGMRES.cpp:113-330;
 * Frommer & Glaessner 1998): restarted GMRES(m) on the seed system A x = b (x
 * from the true residual b - A x at every restart), every shift's residual kept
 * collinear with the seed's: with z = beta e_1 - Hbar y, shift n solves
 * [Hbar + c_n I~ | z] (y_n; beta0_n') = beta0_n beta e_1 and adds V y_n.
 * Stop when max |beta0_n| < accuracy * blen (blen = |b|^2, or 1 absolute),
 * the reference's rule.  The small systems by Gaussian elimination with
 * partial pivoting (the reference: Givens / QR on the device; same solutions). */
static int solve_square(int n, cplx* A, cplx* rhs, cplx* out) {   /* A n x n row-major, destroyed */
    for (int col = 0; col < n; ++col) {
        int piv = col;
        for (int r = col + 1; r < n; ++r) if (cabs(A[r * n + col]) > cabs(A[piv * n + col])) piv = r;
        if (cabs(A[piv * n + col]) == 0.0) return 0;
        if (piv != col) {
            for (int c = 0; c < n; ++c) { cplx t = A[col * n + c]; A[col * n + c] = A[piv * n + c]; A[piv * n + c] = t; }
            cplx t = rhs[col]; rhs[col] = rhs[piv]; rhs[piv] = t;
        }
        for (int r = col + 1; r < n; ++r) {
            const cplx f = A[r * n + col] / A[col * n + col];
            if (f == 0) continue;
            for (int c = col; c < n; ++c) A[r * n + c] -= f * A[col * n + c];
            rhs[r] -= f * rhs[col];
        }
    }
    for (int r = n - 1; r >= 0; --r) {
        cplx acc = rhs[r];
        for (int c = r + 1; c < n; ++c) acc -= A[r * n + c] * out[c];
        out[r] = acc / A[r * n + r];
    }
    return 1;
}

int clgo_gmres_ms(const clgo_op* op, const double* b, int nshift, const double* shifts_c, double* x,
                  int maxdim, int restart, double accuracy, int absolute, clgo_info* info) {
    const long n = clgo_op_len(op);
    const int m = maxdim;
    double** v = (double**)malloc(sizeof(double*) * m);
    for (int i = 0; i < m; ++i) v[i] = valloc(n);
    double *W = valloc(n), *X = valloc(n), *T = valloc(n);
    cplx* h = (cplx*)calloc((size_t)(m + 1) * m, sizeof(cplx));
    cplx* hh = (cplx*)calloc((size_t)(m + 1) * (m + 1), sizeof(cplx));
    cplx *y = (cplx*)calloc((size_t)m + 1, sizeof(cplx)), *z = (cplx*)calloc((size_t)m + 1, sizeof(cplx)),
         *g = (cplx*)calloc((size_t)m + 1, sizeof(cplx)), *w = (cplx*)calloc((size_t)m + 1, sizeof(cplx));
    cplx* beta0 = (cplx*)malloc(sizeof(cplx) * nshift);
    for (int s = 0; s < nshift; ++s) beta0[s] = 1;
    const double blen = absolute ? 1.0 : clgo_norm2(n, b);
    memset(x, 0, sizeof(double) * 2 * n * nshift);
    memset(X, 0, sizeof(double) * 2 * n);
    int napply = 0, converged = 0, cycles = 0;
    double maxerr = 0;
    for (int it = 0; it < restart; ++it) {
        ++cycles;
        if (it == 0) vcopy(n, b, v[0]);
        else {
            clgo_apply(op, X, T); ++napply;
#pragma omp parallel for schedule(static)
            for (long k = 0; k < 2 * n; ++k) v[0][k] = b[k] - T[k];
        }
        const double beta = sqrt(clgo_norm2(n, v[0]));
        cscale(n, 1.0 / beta, v[0]);
        for (int j = 0; j < m; ++j) {
            clgo_apply(op, v[j], W); ++napply;
            for (int k = 0; k <= j; ++k) {
                const cplx d = cdot(n, v[k], W);
                h[k * m + j] = d;
                caxpy(n, -d, v[k], W);
            }
            const double wn = sqrt(clgo_norm2(n, W));
            h[(j + 1) * m + j] = wn;
            if (j < m - 1) { cscale(n, 1.0 / wn, W); vcopy(n, W, v[j + 1]); }
        }
        /* the seed: least squares min |beta e1 - Hbar y| through the normal
         * equations of the small problem (Hbar^+ Hbar y = Hbar^+ beta e1) */
        {
            cplx* A = (cplx*)calloc((size_t)m * m, sizeof(cplx));
            for (int r = 0; r < m; ++r) {
                for (int c = 0; c < m; ++c) {
                    cplx acc = 0;
                    for (int k = 0; k <= m; ++k) acc += conj(h[k * m + r]) * h[k * m + c];
                    A[r * m + c] = acc;
                }
                g[r] = conj(h[r]) * beta;   /* (Hbar^+ beta e1)_r = conj(h[0][r]) beta */
            }
            solve_square(m, A, g, y);
            free(A);
        }
        for (int j = 0; j < m; ++j) caxpy(n, y[j], v[j], X);
        for (int r = 0; r <= m; ++r) {
            cplx hy = 0;
            for (int c = 0; c < m; ++c) hy += h[r * m + c] * y[c];
            z[r] = (r == 0 ? beta : 0.0) - hy;
        }
        maxerr = 0;
        for (int s = 0; s < nshift; ++s) {
            const cplx cs = shifts_c[2 * s] + I * shifts_c[2 * s + 1];
            for (int r = 0; r <= m; ++r) {
                for (int c = 0; c < m; ++c) hh[r * (m + 1) + c] = h[r * m + c] + (r == c ? cs : 0.0);
                hh[r * (m + 1) + m] = z[r];
                g[r] = (r == 0) ? beta0[s] * beta : 0.0;
            }
            solve_square(m + 1, hh, g, w);
            beta0[s] = w[m];
            if (cabs(beta0[s]) > maxerr) maxerr = cabs(beta0[s]);
            for (int j = 0; j < m; ++j) caxpy(n, w[j], v[j], x + 2 * n * s);
        }
        if (maxerr < accuracy * blen) { converged = 1; break; }
    }
    if (info) {
        info->iterations = napply; info->restarts = cycles; info->converged = converged;
        info->last_deviation = maxerr;
        double worst = 0;
        for (int s = 0; s < nshift; ++s) {
            const double t = clgo_true_residual(op, b, x + 2 * n * s, shifts_c[2 * s], shifts_c[2 * s + 1]);
            if (t > worst) worst = t;
        }
        info->true_rel_residual = worst;
    }
    for (int i = 0; i < m; ++i) free(v[i]);
    free(v); free(W); free(X); free(T); free(h); free(hh); free(y); free(z); free(g); free(w); free(beta0);
    return converged;
}
