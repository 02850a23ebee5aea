/*
 * fp4_oracle.c -- CPU restatement of FourPhonon's scattering-rate hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product path
 * and the timed CPU baseline of bench.py.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it.  The product library never links
 * or calls it.
 *
 * Every routine below restates one reference routine line by line, in the same
 * loop order and with the same floating-point operation order (compile with
 * -O2 -ffp-contract=off so that no multiply-add is fused).  Citations are to
 * the reference source tree (FourPhonon, Src/...).
 *
 * Conventions (identical to the Fortran arrays passed through the C-ABI):
 *   energy(nptk,nb)           energy[b*nptk + q]
 *   velocity(nptk,nb,3)       velocity[(d*nb + b)*nptk + q]
 *   eigenvect(nptk,nb,nb)     complex, eig[2*((c*nb + b)*nptk + q)] (+1 = imag)
 *   IJK(3,nptk)               ijk[3*q + d]
 *   List(Nlist)               1-based q-point indices
 *   Phi(3,3,3,Ntri)           phi[((c*3 + r)*3 + s)*3 + t] == Phi(t,s,r,c)
 *   Psi(3,3,3,3,Ntri)         psi[(((c*3 + r)*3 + s)*3 + t)*3 + u] == Psi(u,t,s,r,c)
 *   R_j(3,Ntri)               rj[3*c + d]
 *   rate(Nb,Nlist)            rate[ll*nb + i]
 * q-point and atom indices stored in arrays are 1-based, exactly as in the
 * reference; loop variables below are 1-based where the reference's are.
 *
 * Single-precision literals.  The CPU reference multiplies by default-REAL
 * literals (5.60626442, 3.37617087, 0.001, 1e22 inside hbarp); these are
 * reproduced below as (double)(float) constants.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* data.f90:5-7 */
#define FP4O_PI 3.141592653589793238
#define FP4O_KB 1.380648813e-23
#define FP4O_HBAR 1.05457172647e-22

typedef struct {
    int ngrid[3];
    int nptk, nb, nlist;
    double rlattvec[9]; /* rlattvec(3,3) column-major: rlattvec[d + 3*n] */
    double scalebroad, T, omega_max;
    int onlyharmonic;
    const double *energy;
    const double *velocity;
    const double *eig; /* interleaved complex */
    const int *list;
    const int *ijk;
    const double *masses; /* masses(nelements) */
    const int *types;     /* types(natoms), 1-based element ids */
} fp4o_sys;

typedef struct {
    int ntri;
    const double *phi; /* 27*ntri (3ph) or 81*ntri (4ph) */
    const double *rj, *rk, *rl;
    const int *ii, *ij, *ik, *il;
} fp4o_ifc;

/* processes.f90:20  hbarp=hbar*1e22 with a default-REAL 1e22 */
static double hbarp(void) { return FP4O_HBAR * (double)1e22f; }

static inline double E(const fp4o_sys *s, int q1, int b1) { return s->energy[(size_t)(b1 - 1) * s->nptk + (q1 - 1)]; }
static inline double Vel(const fp4o_sys *s, int q1, int b1, int d) {
    return s->velocity[((size_t)d * s->nb + (b1 - 1)) * s->nptk + (q1 - 1)];
}
static inline void Eig(const fp4o_sys *s, int q1, int b1, int c1, double *re, double *im) {
    size_t o = 2 * (((size_t)(c1 - 1) * s->nb + (b1 - 1)) * s->nptk + (q1 - 1));
    *re = s->eig[o];
    *im = s->eig[o + 1];
}

/* config.f90:481-499 base_sigma: max-of-three form, then sqrt(x/2.) */
double fp4o_base_sigma(const fp4o_sys *s, const double v[3]) {
    double m[3];
    for (int nu = 0; nu < 3; nu++) {
        const double *r = s->rlattvec + 3 * nu;
        double dp = 0.0;
        dp = dp + r[0] * v[0];
        dp = dp + r[1] * v[1];
        dp = dp + r[2] * v[2];
        double x = dp / (double)s->ngrid[nu];
        m[nu] = x * x;
    }
    double b = m[0];
    if (m[1] > b) b = m[1];
    if (m[2] > b) b = m[2];
    return sqrt(b / 2.0);
}

static double sigma_of(const fp4o_sys *s, int qa, int ba, int qb, int bb) {
    double v[3];
    for (int d = 0; d < 3; d++) v[d] = Vel(s, qa, ba, d) - Vel(s, qb, bb, d);
    return s->scalebroad * fp4o_base_sigma(s, v);
}

/* Index_N(i,j,k)=(k*Ngrid(2)+j)*Ngrid(1)+i+1 (processes.f90:384-390) */
static inline int index_n(const fp4o_sys *s, const int q[3]) {
    return (q[2] * s->ngrid[1] + q[1]) * s->ngrid[0] + q[0] + 1;
}
static inline int fmodulo(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}
/* realq=matmul(rlattvec,q/dble(ngrid)) */
static void realq(const fp4o_sys *s, const int q[3], double out[3]) {
    double x[3];
    for (int d = 0; d < 3; d++) x[d] = (double)q[d] / (double)s->ngrid[d];
    for (int i = 0; i < 3; i++) {
        double acc = 0.0;
        acc = acc + s->rlattvec[i + 0] * x[0];
        acc = acc + s->rlattvec[i + 3] * x[1];
        acc = acc + s->rlattvec[i + 6] * x[2];
        out[i] = acc;
    }
}
static inline double dot3(const double *a, const double *b) {
    double acc = 0.0;
    acc = acc + a[0] * b[0];
    acc = acc + a[1] * b[1];
    acc = acc + a[2] * b[2];
    return acc;
}
static inline double fbe(const fp4o_sys *s, double w) { return 1.0 / (exp(FP4O_HBAR * w / FP4O_KB / s->T) - 1.0); }

/* ------------------------------------------------------------------------- */
/* Matrix elements                                                            */
/* ------------------------------------------------------------------------- */

/* processes.f90:25-81 (Vp_plus, which=+1) and 84-139 (Vp_minus, which=-1). */
void fp4o_vp3(const fp4o_sys *s, const fp4o_ifc *f, int which, int i, int j, int k, int q, int qp, int qdp,
              const double rqp[3], const double rqdp[3], double *out_re, double *out_im) {
    double vre = 0.0, vim = 0.0;
    for (int ll = 0; ll < f->ntri; ll++) {
        double m = s->masses[s->types[f->ii[ll] - 1] - 1] * s->masses[s->types[f->ij[ll] - 1] - 1] *
                   s->masses[s->types[f->ik[ll] - 1] - 1];
        double r = 1.0 / sqrt(m);
        double a1 = (which > 0 ? 1.0 : -1.0) * dot3(rqp, f->rj + 3 * ll);
        double a2 = -dot3(rqdp, f->rk + 3 * ll);
        double c1r = cos(a1), c1i = sin(a1), c2r = cos(a2), c2i = sin(a2);
        /* prefactor = r * phexp(a1) * phexp(a2) */
        double p1r = r * c1r, p1i = r * c1i;
        double pr = p1r * c2r - p1i * c2i, pi = p1r * c2i + p1i * c2r;
        double v0r = 0.0, v0i = 0.0;
        for (int rr = 1; rr <= 3; rr++)
            for (int ss = 1; ss <= 3; ss++)
                for (int tt = 1; tt <= 3; tt++) {
                    double ph = f->phi[((ll * 3 + (rr - 1)) * 3 + (ss - 1)) * 3 + (tt - 1)];
                    double e1r, e1i, e2r, e2i, e3r, e3i;
                    Eig(s, q, i, tt + 3 * (f->ii[ll] - 1), &e1r, &e1i);
                    Eig(s, qp, j, ss + 3 * (f->ij[ll] - 1), &e2r, &e2i);
                    Eig(s, qdp, k, rr + 3 * (f->ik[ll] - 1), &e3r, &e3i);
                    if (which < 0) e2i = -e2i;
                    e3i = -e3i;
                    double ar = ph * e1r, ai = ph * e1i;
                    double br = ar * e2r - ai * e2i, bi = ar * e2i + ai * e2r;
                    double cr = br * e3r - bi * e3i, ci = br * e3i + bi * e3r;
                    v0r = v0r + cr;
                    v0i = v0i + ci;
                }
        vre = vre + (pr * v0r - pi * v0i);
        vim = vim + (pr * v0i + pi * v0r);
    }
    *out_re = vre;
    *out_im = vim;
}

/* processes.f90:142-330 Vp_pp (ch=0), Vp_pm (ch=1), Vp_mm (ch=2). */
void fp4o_vp4(const fp4o_sys *s, const fp4o_ifc *f, int ch, int i, int j, int k, int l, int q, int qp, int qdp,
              int qtp, const double rqp[3], const double rqdp[3], const double rqtp[3], double *out_re,
              double *out_im) {
    /* sign of the q' and q'' phases, and which eigenvectors are conjugated */
    double sj = (ch == 2) ? -1.0 : 1.0;
    double sk = (ch == 0) ? 1.0 : -1.0;
    int conj_j = (ch == 2), conj_k = (ch != 0);
    double vre = 0.0, vim = 0.0;
    for (int ll = 0; ll < f->ntri; ll++) {
        double m = s->masses[s->types[f->ii[ll] - 1] - 1] * s->masses[s->types[f->ij[ll] - 1] - 1] *
                   s->masses[s->types[f->ik[ll] - 1] - 1] * s->masses[s->types[f->il[ll] - 1] - 1];
        double r = 1.0 / sqrt(m);
        double a1 = sj * dot3(rqp, f->rj + 3 * ll);
        double a2 = sk * dot3(rqdp, f->rk + 3 * ll);
        double a3 = -dot3(rqtp, f->rl + 3 * ll);
        double c1r = cos(a1), c1i = sin(a1), c2r = cos(a2), c2i = sin(a2), c3r = cos(a3), c3i = sin(a3);
        double p1r = r * c1r, p1i = r * c1i;
        double p2r = p1r * c2r - p1i * c2i, p2i = p1r * c2i + p1i * c2r;
        double pr = p2r * c3r - p2i * c3i, pi = p2r * c3i + p2i * c3r;
        double v0r = 0.0, v0i = 0.0;
        for (int rr = 1; rr <= 3; rr++)
            for (int ss = 1; ss <= 3; ss++)
                for (int tt = 1; tt <= 3; tt++)
                    for (int uu = 1; uu <= 3; uu++) {
                        double ph = f->phi[(((ll * 3 + (rr - 1)) * 3 + (ss - 1)) * 3 + (tt - 1)) * 3 + (uu - 1)];
                        double e1r, e1i, e2r, e2i, e3r, e3i, e4r, e4i;
                        Eig(s, q, i, uu + 3 * (f->ii[ll] - 1), &e1r, &e1i);
                        Eig(s, qp, j, tt + 3 * (f->ij[ll] - 1), &e2r, &e2i);
                        Eig(s, qdp, k, ss + 3 * (f->ik[ll] - 1), &e3r, &e3i);
                        Eig(s, qtp, l, rr + 3 * (f->il[ll] - 1), &e4r, &e4i);
                        if (conj_j) e2i = -e2i;
                        if (conj_k) e3i = -e3i;
                        e4i = -e4i;
                        double ar = ph * e1r, ai = ph * e1i;
                        double br = ar * e2r - ai * e2i, bi = ar * e2i + ai * e2r;
                        double cr = br * e3r - bi * e3i, ci = br * e3i + bi * e3r;
                        double dr = cr * e4r - ci * e4i, di = cr * e4i + ci * e4r;
                        v0r = v0r + dr;
                        v0i = v0i + di;
                    }
        vre = vre + (pr * v0r - pi * v0i);
        vim = vim + (pr * v0i + pi * v0r);
    }
    *out_re = vre;
    *out_im = vim;
}

/* ------------------------------------------------------------------------- */
/* Three-phonon processes                                                     */
/* ------------------------------------------------------------------------- */

/*
 * One mode of NP_plus/NP_minus (processes.f90:712-823), Ind_only_plus/minus
 * (1074-1192) or RTA_plus/RTA_minus (1313-1471), selected by `mode`:
 *   mode 0: count + phase space (NP_*; loop ii outer, j inner)
 *   mode 1: index lists (Ind_only_*; loop j outer, ii inner)
 *   mode 2: RTA rate (RTA_*; loop ii outer, j inner)
 *   mode 3: per-process Gamma + index lists (Ind_plus/Ind_minus 361-521; j outer)
 * which = +1 absorption, -1 emission.
 */
typedef struct {
    int64_t n;
    double P, gamma, wp;
    int64_t cap;
    int32_t *ind2, *ind3;
    double *g;
} acc3_t;

static void proc3_one(const fp4o_sys *s, const fp4o_ifc *f, int mm, int which, int mode, acc3_t *a) {
    const int nb = s->nb, nptk = s->nptk;
    int i = (mm - 1) % nb + 1;
    int ll = (mm - 1) / nb + 1;
    int q[3];
    for (int d = 0; d < 3; d++) q[d] = s->ijk[3 * (s->list[ll - 1] - 1) + d];
    double omega = E(s, s->list[ll - 1], i);
    a->n = 0;
    a->P = 0.0;
    a->gamma = 0.0;
    a->wp = 0.0;
    double hp = hbarp();
    if (omega != 0) {
        int outer_j = (mode == 1 || mode == 3);
        int n_out = outer_j ? nb : nptk, n_in = outer_j ? nptk : nb;
        for (int o = 1; o <= n_out; o++)
            for (int in = 1; in <= n_in; in++) {
                int ii = outer_j ? in : o;
                int j = outer_j ? o : in;
                int qp[3], qdp[3];
                for (int d = 0; d < 3; d++) qp[d] = s->ijk[3 * (ii - 1) + d];
                double rqp[3];
                realq(s, qp, rqp);
                double omegap = E(s, ii, j);
                double fbep = (mode >= 2) ? fbe(s, omegap) : 0.0;
                for (int k = 1; k <= nb; k++) {
                    for (int d = 0; d < 3; d++) qdp[d] = fmodulo(q[d] + which * qp[d], s->ngrid[d]);
                    int ss = index_n(s, qdp);
                    double omegadp = E(s, ss, k);
                    if ((omegap != 0) && (omegadp != 0)) {
                        double sigma = sigma_of(s, ii, j, ss, k);
                        double delta = (which > 0) ? (omega + omegap - omegadp) : (omega - omegap - omegadp);
                        if (fabs(delta) <= 2.0 * sigma) {
                            if (mode == 0) {
                                a->n++;
                                a->P = a->P + exp(-(delta * delta) / (sigma * sigma)) /
                                                  (sigma * sqrt(FP4O_PI) * (double)(nptk * nptk) * (double)(nb * nb * nb));
                                continue;
                            }
                            if (mode == 1 || mode == 3) {
                                if (a->n < a->cap) {
                                    a->ind2[a->n] = (ii - 1) * nb + j;
                                    a->ind3[a->n] = (ss - 1) * nb + k;
                                }
                            }
                            if (mode == 1) {
                                a->n++;
                                continue;
                            }
                            double fbedp = fbe(s, omegadp);
                            double bose = (which > 0) ? (fbep - fbedp) : (fbep + fbedp + 1);
                            double wp3 = bose * exp(-(delta * delta) / (sigma * sigma)) / sigma / sqrt(FP4O_PI) /
                                         (omega * omegap * omegadp);
                            a->wp = a->wp + wp3;
                            if (mode == 3) {
                                double rqdp[3];
                                realq(s, qdp, rqdp);
                                double vr, vi;
                                fp4o_vp3(s, f, which, i, j, k, s->list[ll - 1], ii, ss, rqp, rqdp, &vr, &vi);
                                double av = hypot(vr, vi);
                                double g = hp * FP4O_PI / 4.0 * wp3 * (av * av);
                                g = g * (double)5.60626442f * 1.e8 / nptk;
                                if (a->n < a->cap) a->g[a->n] = g;
                                a->n++;
                                continue;
                            }
                            if (!s->onlyharmonic) {
                                double rqdp[3];
                                realq(s, qdp, rqdp);
                                double vr, vi;
                                fp4o_vp3(s, f, which, i, j, k, s->list[ll - 1], ii, ss, rqp, rqdp, &vr, &vi);
                                double av = hypot(vr, vi);
                                a->gamma = a->gamma + hp * FP4O_PI / 4.0 * wp3 * (av * av);
                            }
                            a->n++;
                        }
                    }
                }
            }
        if (mode >= 2) {
            if (which > 0)
                a->wp = a->wp / nptk;
            else
                a->wp = a->wp * 5.e-1 / nptk;
        }
    }
    if (mode == 2) a->gamma = a->gamma * (double)5.60626442f * 1.e8 / nptk;
}

static int gate(const fp4o_sys *s, int mm) {
    int i = (mm - 1) % s->nb + 1, ll = (mm - 1) / s->nb + 1;
    return E(s, s->list[ll - 1], i) <= s->omega_max;
}

/* NP_driver (processes.f90:983-1067) over modes [mm0,mm1) (0-based). */
void fp4o_np3(const fp4o_sys *s, int mm0, int mm1, int32_t *n_plus, int32_t *n_minus, double *p_plus,
              double *p_minus) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int m0 = mm0; m0 < mm1; m0++) {
        int mm = m0 + 1;
        acc3_t a;
        memset(&a, 0, sizeof a);
        n_plus[m0] = n_minus[m0] = 0;
        p_plus[m0] = p_minus[m0] = 0.0;
        if (!gate(s, mm)) continue;
        proc3_one(s, NULL, mm, +1, 0, &a);
        n_plus[m0] = (int32_t)a.n;
        p_plus[m0] = a.P;
        proc3_one(s, NULL, mm, -1, 0, &a);
        n_minus[m0] = (int32_t)a.n;
        p_minus[m0] = a.P;
    }
}

/* Ind_only_plus / Ind_only_minus for one mode (1-based mm).  Returns the count. */
int64_t fp4o_ind_only3(const fp4o_sys *s, int mm, int which, int64_t cap, int32_t *ind2, int32_t *ind3) {
    acc3_t a;
    memset(&a, 0, sizeof a);
    a.cap = cap;
    a.ind2 = ind2;
    a.ind3 = ind3;
    proc3_one(s, NULL, mm, which, 1, &a);
    return a.n;
}

/* RTA_driver (processes.f90:1676-1775): rate_minus carries the driver's x0.5. */
void fp4o_rta3(const fp4o_sys *s, const fp4o_ifc *f, int mm0, int mm1, double *rate_plus, double *rate_minus,
               double *wp3_plus, double *wp3_minus) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int m0 = mm0; m0 < mm1; m0++) {
        int mm = m0 + 1;
        acc3_t a;
        memset(&a, 0, sizeof a);
        rate_plus[m0] = rate_minus[m0] = wp3_plus[m0] = wp3_minus[m0] = 0.0;
        if (!gate(s, mm)) continue;
        proc3_one(s, f, mm, +1, 2, &a);
        rate_plus[m0] = a.gamma;
        wp3_plus[m0] = a.wp;
        proc3_one(s, f, mm, -1, 2, &a);
        rate_minus[m0] = a.gamma * 5.e-1;
        wp3_minus[m0] = a.wp;
    }
}

/*
 * Ind_driver (processes.f90:524-707): per-process Gamma lists in the order of
 * Ind_plus/Ind_minus, laid out at the Naccum offsets of N_plus/N_minus.
 * rate_minus carries the x0.5; Gamma_minus does not (iterations.f90 applies it).
 */
void fp4o_ind3(const fp4o_sys *s, const fp4o_ifc *f, const int32_t *n_plus, const int32_t *n_minus,
               int32_t *ind2_p, int32_t *ind3_p, double *gamma_p, int32_t *ind2_m, int32_t *ind3_m,
               double *gamma_m, double *rate_plus, double *rate_minus, double *wp3_plus, double *wp3_minus) {
    int nm = s->nb * s->nlist;
    int64_t *acc_p = (int64_t *)malloc(sizeof(int64_t) * (nm + 1));
    int64_t *acc_m = (int64_t *)malloc(sizeof(int64_t) * (nm + 1));
    acc_p[0] = acc_m[0] = 0;
    for (int m = 0; m < nm; m++) {
        acc_p[m + 1] = acc_p[m] + n_plus[m];
        acc_m[m + 1] = acc_m[m] + n_minus[m];
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int m0 = 0; m0 < nm; m0++) {
        int mm = m0 + 1;
        acc3_t a;
        rate_plus[m0] = rate_minus[m0] = wp3_plus[m0] = wp3_minus[m0] = 0.0;
        if (n_plus[m0] != 0) {
            memset(&a, 0, sizeof a);
            a.cap = n_plus[m0];
            a.ind2 = ind2_p + acc_p[m0];
            a.ind3 = ind3_p + acc_p[m0];
            a.g = gamma_p + acc_p[m0];
            proc3_one(s, f, mm, +1, 3, &a);
            wp3_plus[m0] = a.wp;
            double sum = 0.0;
            for (int64_t x = 0; x < n_plus[m0]; x++) sum = sum + a.g[x];
            rate_plus[m0] = sum;
        }
        if (n_minus[m0] != 0) {
            memset(&a, 0, sizeof a);
            a.cap = n_minus[m0];
            a.ind2 = ind2_m + acc_m[m0];
            a.ind3 = ind3_m + acc_m[m0];
            a.g = gamma_m + acc_m[m0];
            proc3_one(s, f, mm, -1, 3, &a);
            wp3_minus[m0] = a.wp;
            double sum = 0.0;
            for (int64_t x = 0; x < n_minus[m0]; x++) sum = sum + a.g[x];
            rate_minus[m0] = sum * 5.e-1;
        }
    }
    free(acc_p);
    free(acc_m);
}

/* ------------------------------------------------------------------------- */
/* Four-phonon processes                                                      */
/* ------------------------------------------------------------------------- */

/*
 * One mode of a four-phonon channel, ch = 0 (++), 1 (+-), 2 (--):
 *   NP_plusplus/plusminus/minusminus  processes.f90:2263-2476   (mode 0)
 *   Ind_only_plusplus/...             processes.f90:2854-3074   (mode 1)
 *   RTA_plusplus/...                  processes.f90:3828-4129   (mode 2)
 *   Ind_plusplus/plusminus/minusminus processes.f90:3254-3548   (mode 3)
 * All four share the loop nest ii, jj, j, k, l with the channel's restrictions.
 */
typedef struct {
    int64_t n;
    double P, gamma, wp;
    int64_t cap;
    int64_t *ind2, *ind3, *ind4;
    double *glist; /* mode 3: Gamma of each listed process */
    int ii0, ii1;  /* optional q' range [ii0, ii1) (0-based); ii1 == 0 means all */
} acc4_t;

static void proc4_one(const fp4o_sys *s, const fp4o_ifc *f, int mm, int ch, int mode, acc4_t *a) {
    const int nb = s->nb, nptk = s->nptk;
    int i = (mm - 1) % nb + 1;
    int ll = (mm - 1) / nb + 1;
    int q[3];
    for (int d = 0; d < 3; d++) q[d] = s->ijk[3 * (s->list[ll - 1] - 1) + d];
    double omega = E(s, s->list[ll - 1], i);
    double hp = hbarp();
    a->n = 0;
    a->P = 0.0;
    a->gamma = 0.0;
    a->wp = 0.0;
    const double floor_sigma = (double)0.001f;
    const double pdenom = (double)nptk * (double)nptk * (double)nptk;
    int ii_lo = (a->ii1 > 0) ? a->ii0 + 1 : 1, ii_hi = (a->ii1 > 0) ? a->ii1 : nptk;
    if (omega != 0) {
        for (int ii = ii_lo; ii <= ii_hi; ii++) {
            int jj0 = (ch == 1) ? 1 : ii;
            for (int jj = jj0; jj <= nptk; jj++) {
                int qp[3], qdp[3], qtp[3];
                for (int d = 0; d < 3; d++) {
                    qp[d] = s->ijk[3 * (ii - 1) + d];
                    qdp[d] = s->ijk[3 * (jj - 1) + d];
                }
                for (int d = 0; d < 3; d++) {
                    int t = (ch == 0) ? (q[d] + qp[d] + qdp[d]) : (ch == 1) ? (q[d] + qp[d] - qdp[d])
                                                                             : (q[d] - qp[d] - qdp[d]);
                    qtp[d] = fmodulo(t, s->ngrid[d]);
                }
                int ss = index_n(s, qtp);
                if (ch == 0 ? !(ss >= 1) : !(ss >= jj)) continue;
                double rqp[3], rqdp[3], rqtp[3];
                if (mode >= 2) {
                    realq(s, qp, rqp);
                    realq(s, qdp, rqdp);
                    realq(s, qtp, rqtp);
                }
                for (int j = 1; j <= nb; j++) {
                    int kstart = 1;
                    if (ch != 1 && jj == ii) kstart = j;
                    for (int k = kstart; k <= nb; k++) {
                        int lstart = 1;
                        if (ch != 0 && ss == jj) lstart = k;
                        for (int l = lstart; l <= nb; l++) {
                            double omegap = E(s, ii, j), omegadp = E(s, jj, k), omegatp = E(s, ss, l);
                            if (!((omegap != 0) && (omegadp != 0) && (omegatp != 0))) continue;
                            double sigma = sigma_of(s, jj, k, ss, l);
                            if (ch == 1) {
                                int ql = s->list[ll - 1];
                                if (!((ql != jj || i != k) && (ql != ss || i != l) && (ii != jj || j != k) &&
                                      (ii != ss || j != l)))
                                    continue;
                            }
                            double delta = (ch == 0) ? (omega + omegap + omegadp - omegatp)
                                           : (ch == 1) ? (omega + omegap - omegadp - omegatp)
                                                       : (omega - omegap - omegadp - omegatp);
                            if (!(fabs(delta) <= sigma)) continue;
                            if (mode == 1) {
                                if (a->n < a->cap) {
                                    a->ind2[a->n] = (int64_t)(ii - 1) * nb + j;
                                    a->ind3[a->n] = (int64_t)(jj - 1) * nb + k;
                                    a->ind4[a->n] = (int64_t)(ss - 1) * nb + l;
                                }
                                a->n++;
                                continue;
                            }
                            if (sigma <= floor_sigma) sigma = 1 / sqrt(FP4O_PI);
                            if (mode == 3) {
                                /* Ind_*: the process's own Gamma, listed in enumeration order */
                                double f1 = fbe(s, omegap), f2 = fbe(s, omegadp), f3 = fbe(s, omegatp);
                                double bose = (ch == 0)   ? (f1 * f2 * (1 + f3) - (1 + f1) * (1 + f2) * f3)
                                              : (ch == 1) ? (f1 * (1 + f2) * (1 + f3) - (1 + f1) * f2 * f3)
                                                          : ((1 + f1) * (1 + f2) * (1 + f3) - f1 * f2 * f3);
                                double wp4 = bose * exp(-(delta * delta) / (sigma * sigma)) / sigma /
                                             sqrt(FP4O_PI) / (omega * omegap * omegadp * omegatp);
                                if (omegap <= 1.25 || omegadp <= 1.25 || omegatp <= 1.25) wp4 = 0;
                                a->wp = a->wp + wp4;
                                double vr, vi;
                                fp4o_vp4(s, f, ch, i, j, k, l, s->list[ll - 1], ii, jj, ss, rqp, rqdp, rqtp, &vr,
                                         &vi);
                                double av = hypot(vr, vi);
                                double g = hp * hp * FP4O_PI / 8.0 * wp4 * (av * av);
                                g = g * (double)3.37617087f * 1.e9 / nptk / nptk;
                                if (a->n < a->cap) {
                                    a->ind2[a->n] = (int64_t)(ii - 1) * nb + j;
                                    a->ind3[a->n] = (int64_t)(jj - 1) * nb + k;
                                    a->ind4[a->n] = (int64_t)(ss - 1) * nb + l;
                                    a->glist[a->n] = g;
                                }
                                a->n++;
                                continue;
                            }
                            a->n++;
                            if (mode == 0) {
                                a->P = a->P + exp(-(delta * delta) / (sigma * sigma)) /
                                                  (sigma * sqrt(FP4O_PI) * pdenom * (double)(nb * nb * nb * nb));
                                continue;
                            }
                            double f1 = fbe(s, omegap), f2 = fbe(s, omegadp), f3 = fbe(s, omegatp);
                            double bose = (ch == 0)   ? (f1 * f2 * (1 + f3) - (1 + f1) * (1 + f2) * f3)
                                          : (ch == 1) ? (f1 * (1 + f2) * (1 + f3) - (1 + f1) * f2 * f3)
                                                      : ((1 + f1) * (1 + f2) * (1 + f3) - f1 * f2 * f3);
                            double wp4 = bose * exp(-(delta * delta) / (sigma * sigma)) / sigma / sqrt(FP4O_PI) /
                                         (omega * omegap * omegadp * omegatp);
                            if (omegap <= 1.25 || omegadp <= 1.25 || omegatp <= 1.25) wp4 = 0;
                            a->wp = a->wp + wp4;
                            if (!s->onlyharmonic) {
                                double vr, vi;
                                fp4o_vp4(s, f, ch, i, j, k, l, s->list[ll - 1], ii, jj, ss, rqp, rqdp, rqtp, &vr,
                                         &vi);
                                double av = hypot(vr, vi);
                                a->gamma = a->gamma + hp * hp * FP4O_PI / 8.0 * wp4 * (av * av);
                            }
                        }
                    }
                }
            }
        }
        if (mode >= 2) a->wp = a->wp / nptk / nptk;
    }
    if (mode == 2) a->gamma = a->gamma * (double)3.37617087f * 1.e9 / nptk / nptk;
}

/* NP_driver_4ph (processes.f90:2749-2847) over modes [mm0,mm1). */
void fp4o_np4(const fp4o_sys *s, int mm0, int mm1, int64_t *n_pp, int64_t *n_pm, int64_t *n_mm, double *p_pp,
              double *p_pm, double *p_mm) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int m0 = mm0; m0 < mm1; m0++) {
        int mm = m0 + 1;
        acc4_t a;
        memset(&a, 0, sizeof a);
        n_pp[m0] = n_pm[m0] = n_mm[m0] = 0;
        p_pp[m0] = p_pm[m0] = p_mm[m0] = 0.0;
        if (!gate(s, mm)) continue;
        proc4_one(s, NULL, mm, 0, 0, &a);
        n_pp[m0] = a.n;
        p_pp[m0] = a.P;
        proc4_one(s, NULL, mm, 1, 0, &a);
        n_pm[m0] = a.n;
        p_pm[m0] = a.P;
        proc4_one(s, NULL, mm, 2, 0, &a);
        n_mm[m0] = a.n;
        p_mm[m0] = a.P;
    }
}

/* Ind_only_plusplus/plusminus/minusminus for one mode; returns the count. */
int64_t fp4o_ind_only4(const fp4o_sys *s, int mm, int ch, int64_t cap, int64_t *ind2, int64_t *ind3,
                       int64_t *ind4) {
    acc4_t a;
    memset(&a, 0, sizeof a);
    a.cap = cap;
    a.ind2 = ind2;
    a.ind3 = ind3;
    a.ind4 = ind4;
    proc4_one(s, NULL, mm, ch, 1, &a);
    return a.n;
}

/* RTA_driver_4ph (processes.f90:5174-5311) over modes [mm0,mm1). */
void fp4o_rta4(const fp4o_sys *s, const fp4o_ifc *f, int mm0, int mm1, double *rate_pp, double *rate_pm,
               double *rate_mm, double *wp_pp, double *wp_pm, double *wp_mm) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int m0 = mm0; m0 < mm1; m0++) {
        int mm = m0 + 1;
        acc4_t a;
        memset(&a, 0, sizeof a);
        rate_pp[m0] = rate_pm[m0] = rate_mm[m0] = wp_pp[m0] = wp_pm[m0] = wp_mm[m0] = 0.0;
        if (!gate(s, mm)) continue;
        proc4_one(s, f, mm, 0, 2, &a);
        rate_pp[m0] = a.gamma;
        wp_pp[m0] = a.wp;
        proc4_one(s, f, mm, 1, 2, &a);
        rate_pm[m0] = a.gamma;
        wp_pm[m0] = a.wp;
        proc4_one(s, f, mm, 2, 2, &a);
        rate_mm[m0] = a.gamma;
        wp_mm[m0] = a.wp;
    }
}

/*
 * Ind_driver_4ph (processes.f90:3551-3822): per-process Gamma lists of the
 * three channels at offsets Naccum(mm) = sum of N(1:mm-1), rate = sum(Gamma0)
 * in list order, WP4 per mode.  Modes with N(mm) == 0 are skipped, as there.
 */
void fp4o_ind4(const fp4o_sys *s, const fp4o_ifc *f, const int64_t *n_pp, const int64_t *n_pm, const int64_t *n_mm,
               int64_t *i2pp, int64_t *i3pp, int64_t *i4pp, double *g_pp, int64_t *i2pm, int64_t *i3pm,
               int64_t *i4pm, double *g_pm, int64_t *i2mm, int64_t *i3mm, int64_t *i4mm, double *g_mm,
               double *rate_pp, double *rate_pm, double *rate_mm, double *wp_pp, double *wp_pm, double *wp_mm) {
    const int nm = s->nb * s->nlist;
    const int64_t *N[3] = {n_pp, n_pm, n_mm};
    int64_t *I2[3] = {i2pp, i2pm, i2mm}, *I3[3] = {i3pp, i3pm, i3mm}, *I4[3] = {i4pp, i4pm, i4mm};
    double *G[3] = {g_pp, g_pm, g_mm}, *R[3] = {rate_pp, rate_pm, rate_mm}, *W[3] = {wp_pp, wp_pm, wp_mm};
    int64_t *acc = (int64_t *)calloc((size_t)3 * (nm + 1), sizeof(int64_t));
    for (int ch = 0; ch < 3; ch++)
        for (int m = 0; m < nm; m++) acc[ch * (nm + 1) + m + 1] = acc[ch * (nm + 1) + m] + N[ch][m];
#pragma omp parallel for schedule(dynamic, 1)
    for (int x = 0; x < 3 * nm; x++) {
        int ch = x % 3, m0 = x / 3;
        R[ch][m0] = 0.0;
        W[ch][m0] = 0.0;
        if (N[ch][m0] == 0) continue;
        int64_t o = acc[ch * (nm + 1) + m0];
        acc4_t a;
        memset(&a, 0, sizeof a);
        a.cap = N[ch][m0];
        a.ind2 = I2[ch] + o;
        a.ind3 = I3[ch] + o;
        a.ind4 = I4[ch] + o;
        a.glist = G[ch] + o;
        proc4_one(s, f, m0 + 1, ch, 3, &a);
        double sum = 0.0;
        for (int64_t e = 0; e < N[ch][m0]; e++) sum = sum + a.glist[e];
        R[ch][m0] = sum;
        W[ch][m0] = a.wp;
    }
    free(acc);
}

/*
 * RTA_driver_4ph restricted to the q' points [ii0,ii1) (0-based): for modes
 * [mm0,mm1) the per-channel rates and WP4 of the processes whose second phonon
 * lies in the range, normalised as the full driver normalises them
 * (processes.f90:3828-4129, 5256).  Summed over a partition of the grid into
 * ranges this is the full RTA_driver_4ph (up to summation order); it checks a
 * large grid where the full sums take too long on the CPU.
 */
void fp4o_rta4_range(const fp4o_sys *s, const fp4o_ifc *f, int mm0, int mm1, int ii0, int ii1, double *rate_pp,
                     double *rate_pm, double *rate_mm, double *wp_pp, double *wp_pm, double *wp_mm) {
    double *R[3] = {rate_pp, rate_pm, rate_mm}, *W[3] = {wp_pp, wp_pm, wp_mm};
#pragma omp parallel for schedule(dynamic, 1)
    for (int x = 0; x < 3 * (mm1 - mm0); x++) {
        int ch = x % 3, m0 = mm0 + x / 3;
        R[ch][m0] = 0.0;
        W[ch][m0] = 0.0;
        if (!gate(s, m0 + 1)) continue;
        acc4_t a;
        memset(&a, 0, sizeof a);
        a.ii0 = ii0;
        a.ii1 = ii1;
        proc4_one(s, f, m0 + 1, ch, 2, &a);
        R[ch][m0] = a.gamma;
        W[ch][m0] = a.wp;
    }
}

/*
 * Timing sample of RTA_driver_4ph spread over the whole workload: the listed
 * modes (0-based), each over the q' points ii_offset, ii_offset + ii_stride,
 * ... (0-based), all three channels.  Returns the number of surviving
 * processes visited; the rates are discarded (timing use only).
 */
int64_t fp4o_rta4_strided(const fp4o_sys *s, const fp4o_ifc *f, const int32_t *modes, int nmodes, int ii_stride,
                          int ii_offset) {
    const int nq = (s->nptk - ii_offset + ii_stride - 1) / ii_stride;
    int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total)
    for (int x = 0; x < nmodes * nq; x++) {
        const int mm = modes[x / nq] + 1, ii = ii_offset + (x % nq) * ii_stride;
        if (!gate(s, mm)) continue;
        for (int ch = 0; ch < 3; ch++) {
            acc4_t a;
            memset(&a, 0, sizeof a);
            a.ii0 = ii;
            a.ii1 = ii + 1;
            proc4_one(s, f, mm, ch, 2, &a);
            total += a.n;
        }
    }
    return total;
}

/*
 * Timing sample of RTA_driver_4ph at the given (mode, q') pairs (0-based), all
 * three channels each.  Returns the number of surviving processes visited; the
 * rates are discarded (timing use only).
 */
int64_t fp4o_rta4_pairs(const fp4o_sys *s, const fp4o_ifc *f, const int32_t *modes, const int32_t *qps, int n) {
    int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total)
    for (int x = 0; x < n; x++) {
        const int mm = modes[x] + 1, ii = qps[x];
        if (!gate(s, mm)) continue;
        for (int ch = 0; ch < 3; ch++) {
            acc4_t a;
            memset(&a, 0, sizeof a);
            a.ii0 = ii;
            a.ii1 = ii + 1;
            proc4_one(s, f, mm, ch, 2, &a);
            total += a.n;
        }
    }
    return total;
}

/*
 * Bounded sample of RTA_driver_4ph for timing: modes [mm0,mm1), each
 * restricted to the q' range [ii0,ii1).  Returns the number of surviving
 * processes visited; rates are not normalised (timing use only).
 */
int64_t fp4o_rta4_sample(const fp4o_sys *s, const fp4o_ifc *f, int mm0, int mm1, int ii0, int ii1) {
    int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total)
    for (int m0 = mm0; m0 < mm1; m0++) {
        int mm = m0 + 1;
        if (!gate(s, mm)) continue;
        for (int ch = 0; ch < 3; ch++) {
            acc4_t a;
            memset(&a, 0, sizeof a);
            a.ii0 = ii0;
            a.ii1 = ii1;
            proc4_one(s, f, mm, ch, 2, &a);
            total += a.n;
        }
    }
    return total;
}

/* ------------------------------------------------------------------------- */
/* Sampled four-phonon estimators                                             */
/* ------------------------------------------------------------------------- */

/* splitmix64 finaliser (Steele, Lea and Flood, OOPSLA 2014). */
static inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* Key of sample n of mode mm (1-based) in channel ch: counter ((mm-1)*3+ch) << 32 | n. */
uint64_t fp4o_sample_base(uint64_t seed, int mm, int ch, int64_t n) {
    uint64_t c = ((uint64_t)((mm - 1) * 3 + ch) << 32) | (uint64_t)n;
    return mix64(seed ^ mix64(c));
}
/* Draw k (0..4) of a sample, uniform on [0, range): high 64 bits of range * u. */
static inline int draw_k(uint64_t base, int k, int range) {
    uint64_t u = mix64(base + (uint64_t)k);
    return (int)(((unsigned __int128)u * (uint64_t)range) >> 64);
}

/*
 * NP_plusplus_sample ... / RTA_plusplus_sample ... (processes.f90:2480-2746,
 * 4811-5172) for modes [mm0, mm1): nsamples uniform draws of (q', j, q'', k, l)
 * per mode and channel, kept when inside the channel's restricted set
 * (++: q''>=q', k>=j if q''=q'; +-: q'''>=q'', l>=k if q'''=q'', pair
 * exclusions; --: both), weighted as the full drivers weight them and scaled by
 * total_process/nsamples.  The draws come from the counter-based stream above
 * in place of the reference's unseeded random_number, and exactly nsamples
 * are drawn.  mode 0: counts and P4 (NP_*_sample); mode 2: Gamma and WP4
 * (RTA_*_sample).  Output arrays are [ch][mode] (3 x nb*nlist).
 */
void fp4o_sample4(const fp4o_sys *s, const fp4o_ifc *f, int mm0, int mm1, int64_t nsamples, uint64_t seed,
                  int mode, int64_t *n_out, double *p_out, double *rate_out, double *wp_out) {
    const int nb = s->nb, nptk = s->nptk, nm = nb * s->nlist;
    const int64_t total = (int64_t)nb * nptk * nb * nptk * nb;
    const double hp = hbarp();
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
    for (int m0 = mm0; m0 < mm1; m0++)
        for (int ch = 0; ch < 3; ch++) {
            const int mm = m0 + 1;
            const int i = (mm - 1) % nb + 1, ll = (mm - 1) / nb + 1;
            int q[3];
            for (int d = 0; d < 3; d++) q[d] = s->ijk[3 * (s->list[ll - 1] - 1) + d];
            const double omega = E(s, s->list[ll - 1], i);
            int64_t n = 0;
            double P = 0.0, gamma = 0.0, wp = 0.0;
            if (gate(s, mm) && omega != 0) {
                for (int64_t it = 0; it < nsamples; it++) {
                    uint64_t base = fp4o_sample_base(seed, mm, ch, it);
                    int ii = draw_k(base, 0, nptk) + 1, j = draw_k(base, 1, nb) + 1;
                    int jj = draw_k(base, 2, nptk) + 1, k = draw_k(base, 3, nb) + 1;
                    int l = draw_k(base, 4, nb) + 1;
                    int qp[3], qdp[3], qtp[3];
                    for (int d = 0; d < 3; d++) {
                        qp[d] = s->ijk[3 * (ii - 1) + d];
                        qdp[d] = s->ijk[3 * (jj - 1) + d];
                        int t = (ch == 0) ? (q[d] + qp[d] + qdp[d]) : (ch == 1) ? (q[d] + qp[d] - qdp[d])
                                                                                 : (q[d] - qp[d] - qdp[d]);
                        qtp[d] = fmodulo(t, s->ngrid[d]);
                    }
                    int ss = index_n(s, qtp);
                    int accept;
                    if (ch == 0)
                        accept = jj >= ii && k >= ((jj == ii) ? j : 1);
                    else if (ch == 1)
                        accept = ss >= jj && l >= ((ss == jj) ? k : 1);
                    else
                        accept = jj >= ii && k >= ((jj == ii) ? j : 1) && ss >= jj && l >= ((ss == jj) ? k : 1);
                    if (!accept) continue;
                    double omegap = E(s, ii, j), omegadp = E(s, jj, k), omegatp = E(s, ss, l);
                    if (!((omegap != 0) && (omegadp != 0) && (omegatp != 0))) continue;
                    double sigma = sigma_of(s, jj, k, ss, l);
                    if (ch == 1) {
                        int ql = s->list[ll - 1];
                        if (!((ql != jj || i != k) && (ql != ss || i != l) && (ii != jj || j != k) &&
                              (ii != ss || j != l)))
                            continue;
                    }
                    double delta = (ch == 0) ? (omega + omegap + omegadp - omegatp)
                                   : (ch == 1) ? (omega + omegap - omegadp - omegatp)
                                               : (omega - omegap - omegadp - omegatp);
                    if (!(fabs(delta) <= sigma)) continue;
                    if (sigma <= (double)0.001f) sigma = 1 / sqrt(FP4O_PI);
                    n++;
                    if (mode == 0) {
                        P = P + exp(-(delta * delta) / (sigma * sigma)) /
                                    (sigma * sqrt(FP4O_PI) * ((double)nptk * (double)nptk * (double)nptk) *
                                     (double)(nb * nb * nb * nb));
                        continue;
                    }
                    double f1 = fbe(s, omegap), f2 = fbe(s, omegadp), f3 = fbe(s, omegatp);
                    double bose = (ch == 0)   ? (f1 * f2 * (1 + f3) - (1 + f1) * (1 + f2) * f3)
                                  : (ch == 1) ? (f1 * (1 + f2) * (1 + f3) - (1 + f1) * f2 * f3)
                                              : ((1 + f1) * (1 + f2) * (1 + f3) - f1 * f2 * f3);
                    double wp4 = bose * exp(-(delta * delta) / (sigma * sigma)) / sigma / sqrt(FP4O_PI) /
                                 (omega * omegap * omegadp * omegatp);
                    if (omegap <= 1.25 || omegadp <= 1.25 || omegatp <= 1.25) wp4 = 0;
                    wp = wp + wp4;
                    if (!s->onlyharmonic) {
                        double rqp[3], rqdp[3], rqtp[3], vr, vi;
                        realq(s, qp, rqp);
                        realq(s, qdp, rqdp);
                        realq(s, qtp, rqtp);
                        fp4o_vp4(s, f, ch, i, j, k, l, s->list[ll - 1], ii, jj, ss, rqp, rqdp, rqtp, &vr, &vi);
                        double av = hypot(vr, vi);
                        gamma = gamma + hp * hp * FP4O_PI / 8.0 * wp4 * (av * av);
                    }
                }
                if (mode == 2) wp = wp / nptk / nptk;
            }
            const size_t o = (size_t)ch * nm + m0;
            if (mode == 0) {
                n_out[o] = (int64_t)((double)n / (double)nsamples * (double)total);
                p_out[o] = P * (double)total / (double)nsamples;
            } else {
                gamma = gamma * (double)3.37617087f * 1.e9 / nptk / nptk;
                rate_out[o] = gamma / (double)nsamples * (double)total;
                wp_out[o] = wp * (double)total / (double)nsamples;
                if (n_out) n_out[o] = n;
            }
        }
}

/* Key of three-phonon sample n of mode mm (1-based) in channel ch (0: absorption,
 * 1: emission): counter (2^30 + (mm-1)*2 + ch) << 32 | n, apart from the 4ph keys. */
uint64_t fp4o_sample3_base(uint64_t seed, int mm, int ch, int64_t n) {
    uint64_t c = ((uint64_t)((1u << 30) + (uint32_t)((mm - 1) * 2 + ch)) << 32) | (uint64_t)n;
    return mix64(seed ^ mix64(c));
}

/*
 * NP_plus_sample / NP_minus_sample (processes.f90:828-979) and RTA_plus_sample /
 * RTA_minus_sample (1474-1672) with the driver's omega_max gate and x0.5 on the
 * emission rate (1735-1760), for modes [mm0, mm1): per mode and channel,
 * nsamples uniform draws of one integer of [1, Nb*nptk*Nb] decoded as the
 * reference decodes rand_num (q' = ii, branches j and k), the q'' of the
 * channel, the 2-sigma test, and the full drivers' weights, scaled by
 * Nb*nptk*Nb/nsamples in the reference's operation order.  The draws come from
 * the counter-based stream above in place of random_number.  mode 0: counts
 * (int32, as N_plus is) and P3; mode 2: Gamma and WP3.  Outputs [ch][mode].
 */
void fp4o_sample3(const fp4o_sys *s, const fp4o_ifc *f, int mm0, int mm1, int64_t nsamples, uint64_t seed,
                  int mode, int32_t *n_out, double *p_out, double *rate_out, double *wp_out) {
    const int nb = s->nb, nptk = s->nptk, nm = nb * s->nlist;
    const int total3 = nb * nptk * nb;
    const double hp = hbarp();
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
    for (int m0 = mm0; m0 < mm1; m0++)
        for (int ch = 0; ch < 2; ch++) {
            const int mm = m0 + 1, which = ch == 0 ? +1 : -1;
            const int i = (mm - 1) % nb + 1, ll = (mm - 1) / nb + 1;
            int q[3];
            for (int d = 0; d < 3; d++) q[d] = s->ijk[3 * (s->list[ll - 1] - 1) + d];
            const double omega = E(s, s->list[ll - 1], i);
            int64_t n = 0;
            double P = 0.0, gamma = 0.0, wp = 0.0;
            const int on = gate(s, mm);
            if (on && omega != 0) {
                for (int64_t it = 0; it < nsamples; it++) {
                    const int rand_num = draw_k(fp4o_sample3_base(seed, mm, ch, it), 0, total3) + 1;
                    const int nn = (rand_num - 1) / nb + 1;
                    const int k = (rand_num - 1) % nb + 1;
                    const int j = (nn - 1) % nb + 1;
                    const int ii = (nn - 1) / nb + 1;
                    int qp[3], qdp[3];
                    for (int d = 0; d < 3; d++) {
                        qp[d] = s->ijk[3 * (ii - 1) + d];
                        qdp[d] = fmodulo(q[d] + which * qp[d], s->ngrid[d]);
                    }
                    const int ss = index_n(s, qdp);
                    const double omegap = E(s, ii, j), omegadp = E(s, ss, k);
                    if (!((omegap != 0) && (omegadp != 0))) continue;
                    const double sigma = sigma_of(s, ii, j, ss, k);
                    const double delta = (which > 0) ? (omega + omegap - omegadp) : (omega - omegap - omegadp);
                    if (!(fabs(delta) <= 2.0 * sigma)) continue;
                    n++;
                    if (mode == 0) {
                        P = P + exp(-(delta * delta) / (sigma * sigma)) /
                                    (sigma * sqrt(FP4O_PI) * (double)(nptk * nptk) * (double)(nb * nb * nb));
                        continue;
                    }
                    const double fbep = fbe(s, omegap), fbedp = fbe(s, omegadp);
                    const double bose = (which > 0) ? (fbep - fbedp) : (fbep + fbedp + 1);
                    const double wp3 = bose * exp(-(delta * delta) / (sigma * sigma)) / sigma / sqrt(FP4O_PI) /
                                       (omega * omegap * omegadp);
                    wp = wp + wp3;
                    if (!s->onlyharmonic) {
                        double rqp[3], rqdp[3], vr, vi;
                        realq(s, qp, rqp);
                        realq(s, qdp, rqdp);
                        fp4o_vp3(s, f, which, i, j, k, s->list[ll - 1], ii, ss, rqp, rqdp, &vr, &vi);
                        const double av = hypot(vr, vi);
                        gamma = gamma + hp * FP4O_PI / 4.0 * wp3 * (av * av);
                    }
                }
                if (mode == 2) wp = (which > 0) ? wp / nptk : wp * 5.e-1 / nptk;
            }
            const size_t o = (size_t)ch * nm + m0;
            if (mode == 0) {
                n_out[o] = on ? (int32_t)((double)n / (double)nsamples * nb * nptk * nb) : 0;
                p_out[o] = on ? P * nb * nptk * nb / (double)nsamples : 0.0;
            } else {
                gamma = gamma * nb * nptk * nb / (double)nsamples;
                gamma = gamma * (double)5.60626442f * 1.e8 / nptk;
                rate_out[o] = on ? ((which > 0) ? gamma : gamma * 5.e-1) : 0.0;
                wp_out[o] = on ? wp * nb * nptk * nb / (double)nsamples : 0.0;
            }
        }
}

/* ------------------------------------------------------------------------- */
/* Iterative BTE and thermal conductivity                                     */
/* ------------------------------------------------------------------------- */

/* iterations.f90:13-30 iteration0.  F_n(nb,nptk,3): F[(d*nptk + q)*nb + b]. */
void fp4o_iteration0(const fp4o_sys *s, int nsymm_rot, const int32_t *nequi, const int32_t *allequi,
                     const double *tau_zero, double *F) {
    for (int ll = 1; ll <= s->nlist; ll++)
        for (int ii = 1; ii <= s->nb; ii++)
            for (int kk = 1; kk <= nequi[ll - 1]; kk++) {
                int qq = allequi[(ll - 1) * nsymm_rot + (kk - 1)];
                for (int d = 0; d < 3; d++)
                    F[((size_t)d * s->nptk + (qq - 1)) * s->nb + (ii - 1)] =
                        tau_zero[(ll - 1) * s->nb + (ii - 1)] * Vel(s, qq, ii, d) * E(s, qq, ii);
            }
}

/* F_n(:,q,:) = transpose(matmul(symmetrizers(:,:,q), transpose(F_n(:,q,:)))) */
static void symmetrize_q(const fp4o_sys *s, const double *symm, double *F, int qq) {
    const double *S = symm + 9 * (size_t)(qq - 1); /* S(a,b) = S[a + 3b] */
    for (int b = 0; b < s->nb; b++) {
        double x[3], y[3];
        for (int d = 0; d < 3; d++) x[d] = F[((size_t)d * s->nptk + (qq - 1)) * s->nb + b];
        for (int a = 0; a < 3; a++) {
            double acc = 0.0;
            acc = acc + S[a + 0] * x[0];
            acc = acc + S[a + 3] * x[1];
            acc = acc + S[a + 6] * x[2];
            y[a] = acc;
        }
        for (int d = 0; d < 3; d++) F[((size_t)d * s->nptk + (qq - 1)) * s->nb + b] = y[d];
    }
}

/*
 * iterations.f90:34-92 iteration (3ph) and 95-215 iteration_4ph: one in-place
 * Gauss-Seidel sweep.  id_equi(nsymm_rot,nptk) is the map of symmetry_map
 * (config.f90:397-419), typeofsym(nsymm_rot,nptk) the wedge's TypeofSymmetry.
 * Pass n_pp == NULL for the 3ph-only sweep.
 */
void fp4o_iteration(const fp4o_sys *s, int nsymm_rot, const int32_t *nequi, const int32_t *allequi,
                    const int32_t *typeofsym, const int32_t *id_equi, const double *symm, const int32_t *n_plus,
                    const int32_t *n_minus, const int32_t *ind2_p, const int32_t *ind3_p, const double *gamma_p,
                    const int32_t *ind2_m, const int32_t *ind3_m, const double *gamma_m, const int64_t *n_pp,
                    const int64_t *n_pm, const int64_t *n_mm, const int64_t *ind2_pp, const int64_t *ind3_pp,
                    const int64_t *ind4_pp, const double *gamma_pp, const int64_t *ind2_pm, const int64_t *ind3_pm,
                    const int64_t *ind4_pm, const double *gamma_pm, const int64_t *ind2_mm,
                    const int64_t *ind3_mm, const int64_t *ind4_mm, const double *gamma_mm,
                    const double *tau_zero, double *F) {
    const int nb = s->nb, nptk = s->nptk;
    double *dF = (double *)calloc((size_t)nb * nptk * 3, sizeof(double));
#define IDQ(sym, q) id_equi[(size_t)((q) - 1) * nsymm_rot + ((sym) - 1)]
#define FN(b, q, d) F[((size_t)(d) * nptk + ((q) - 1)) * nb + ((b) - 1)]
#define DF(b, q, d) dF[((size_t)(d) * nptk + ((q) - 1)) * nb + ((b) - 1)]
    int64_t a_p = 0, a_m = 0, a_pp = 0, a_pm = 0, a_mm = 0;
    for (int ll = 1; ll <= s->nlist; ll++)
        for (int i = 1; i <= nb; i++) {
            int mm = (ll - 1) * nb + i;
            if (mm != 1) {
                a_p += n_plus[mm - 2];
                a_m += n_minus[mm - 2];
                if (n_pp) {
                    a_pp += n_pp[mm - 2];
                    a_pm += n_pm[mm - 2];
                    a_mm += n_mm[mm - 2];
                }
            }
            for (int kk = 1; kk <= nequi[ll - 1]; kk++) {
                int qq = allequi[(ll - 1) * nsymm_rot + (kk - 1)];
                int sym = typeofsym[(ll - 1) * nsymm_rot + (kk - 1)];
                for (int64_t jj = 1; jj <= n_plus[mm - 1]; jj++) {
                    int32_t x2 = ind2_p[a_p + jj - 1], x3 = ind3_p[a_p + jj - 1];
                    int j = (x2 - 1) % nb + 1, m2 = (x2 - 1) / nb + 1;
                    int k = (x3 - 1) % nb + 1, n3 = (x3 - 1) / nb + 1;
                    for (int d = 0; d < 3; d++)
                        DF(i, qq, d) = DF(i, qq, d) + gamma_p[a_p + jj - 1] * (FN(k, IDQ(sym, n3), d) -
                                                                               FN(j, IDQ(sym, m2), d));
                }
                for (int64_t jj = 1; jj <= n_minus[mm - 1]; jj++) {
                    int32_t x2 = ind2_m[a_m + jj - 1], x3 = ind3_m[a_m + jj - 1];
                    int j = (x2 - 1) % nb + 1, m2 = (x2 - 1) / nb + 1;
                    int k = (x3 - 1) % nb + 1, n3 = (x3 - 1) / nb + 1;
                    for (int d = 0; d < 3; d++)
                        DF(i, qq, d) = DF(i, qq, d) + gamma_m[a_m + jj - 1] *
                                                          (FN(k, IDQ(sym, n3), d) + FN(j, IDQ(sym, m2), d)) * 5.e-1;
                }
                if (n_pp) {
                    const int64_t *I2[3] = {ind2_pp, ind2_pm, ind2_mm}, *I3[3] = {ind3_pp, ind3_pm, ind3_mm},
                                  *I4[3] = {ind4_pp, ind4_pm, ind4_mm};
                    const double *G[3] = {gamma_pp, gamma_pm, gamma_mm};
                    const int64_t *NN[3] = {n_pp, n_pm, n_mm};
                    int64_t A[3] = {a_pp, a_pm, a_mm};
                    for (int ch = 0; ch < 3; ch++)
                        for (int64_t jj = 1; jj <= NN[ch][mm - 1]; jj++) {
                            int64_t x2 = I2[ch][A[ch] + jj - 1], x3 = I3[ch][A[ch] + jj - 1],
                                    x4 = I4[ch][A[ch] + jj - 1];
                            int j = (int)((x2 - 1) % nb) + 1, m2 = (int)((x2 - 1) / nb) + 1;
                            int k = (int)((x3 - 1) % nb) + 1, n3 = (int)((x3 - 1) / nb) + 1;
                            int l = (int)((x4 - 1) % nb) + 1, s4 = (int)((x4 - 1) / nb) + 1;
                            double g = G[ch][A[ch] + jj - 1];
                            for (int d = 0; d < 3; d++) {
                                double fl = FN(l, IDQ(sym, s4), d), fj = FN(j, IDQ(sym, m2), d),
                                       fk = FN(k, IDQ(sym, n3), d);
                                double t = (ch == 0) ? (fl - fj - fk) : (ch == 1) ? (fl - fj + fk) : (fl + fj + fk);
                                DF(i, qq, d) = DF(i, qq, d) + g * t;
                            }
                        }
                }
                double tz = tau_zero[(ll - 1) * nb + (i - 1)];
                for (int d = 0; d < 3; d++)
                    FN(i, qq, d) = tz * Vel(s, qq, i, d) * E(s, qq, i) + tz * DF(i, qq, d);
                symmetrize_q(s, symm, F, qq);
            }
        }
#undef IDQ
#undef FN
#undef DF
    free(dF);
}

/* F_n(:,ll,:) symmetrisation over all q (ShengBTE.f90:1288-1290). */
void fp4o_symmetrize_fn(const fp4o_sys *s, const double *symm, double *F) {
    for (int q = 1; q <= s->nptk; q++) symmetrize_q(s, symm, F, q);
}

/*
 * conductivity.f90:11-37 TConduct.  kappa(nb,3,3): kappa[(d2*3 + d1)*nb + b].
 * V is the unit-cell volume in nm^3 (config.f90:243).
 */
void fp4o_tconduct(const fp4o_sys *s, double V, const double *F, double *kappa) {
    const int nb = s->nb, nptk = s->nptk;
    for (int x = 0; x < nb * 9; x++) kappa[x] = 0.0;
    for (int jj = 1; jj <= nb; jj++)
        for (int ii = 2; ii <= nptk; ii++) {
            double tmp[3][3];
            for (int d1 = 0; d1 < 3; d1++)
                for (int d2 = 0; d2 < 3; d2++)
                    tmp[d1][d2] = Vel(s, ii, jj, d1) * F[((size_t)d2 * nptk + (ii - 1)) * nb + (jj - 1)];
            double w = E(s, ii, jj);
            double f = 1.0 / (exp(FP4O_HBAR * w / FP4O_KB / s->T) - 1.0);
            for (int d1 = 0; d1 < 3; d1++)
                for (int d2 = 0; d2 < 3; d2++) {
                    double mode = f * (f + 1) * w * tmp[d1][d2];
                    kappa[(d2 * 3 + d1) * nb + (jj - 1)] = kappa[(d2 * 3 + d1) * nb + (jj - 1)] + mode;
                }
        }
    /* 1e21*hbar**2*ThConductivity/(kB*T*T*V*nptk); 1e21 is a default-REAL literal */
    double fac = (double)1e21f * (FP4O_HBAR * FP4O_HBAR);
    double den = FP4O_KB * s->T * s->T * V * nptk;
    for (int x = 0; x < nb * 9; x++) kappa[x] = fac * kappa[x] / den;
}

/* Euclidean norm of a 3-vector by the scaled sum of squares of reference BLAS dnrm2. */
static double nrm2_3(const double x[3]) {
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < 3; i++) {
        if (x[i] != 0.0) {
            double a = fabs(x[i]);
            if (scale < a) {
                ssq = 1.0 + ssq * (scale / a) * (scale / a);
                scale = a;
            } else {
                ssq = ssq + (a / scale) * (a / scale);
            }
        }
    }
    return scale * sqrt(ssq);
}

/*
 * conductivity.f90:64-97 CumulativeTConduct (omega_mode 0: thresholds on the
 * mean free path, ticks 10**(8(i-1)/(nticks-1)-2) nm evaluated in default
 * REAL as there) and 100-148 CumulativeTConductOmega (omega_mode 1:
 * thresholds on omega, ticks emin+(emax-emin)*i/nticks with emax*1.1).
 * results(nb,3,3,nticks): results[((k*3 + d2)*3 + d1)*nb + b].
 */
void fp4o_cumulative_tconduct(const fp4o_sys *s, double V, const double *F, int nticks, int omega_mode,
                              double *ticks, double *results) {
    const int nb = s->nb, nptk = s->nptk;
    if (omega_mode == 0) {
        for (int ii = 1; ii <= nticks; ii++)
            ticks[ii - 1] = (double)powf(10.0f, 8.0f * ((float)ii - 1.0f) / ((float)nticks - 1.0f) - 2.0f);
    } else {
        double emin = 1.e10, emax = -1.e10;
        for (int ii = 1; ii <= nptk; ii++)
            for (int jj = 1; jj <= nb; jj++) {
                emin = fmin(emin, E(s, ii, jj));
                emax = fmax(emax, E(s, ii, jj));
            }
        emax = emax * 1.1;
        for (int ii = 1; ii <= nticks; ii++) ticks[ii - 1] = emin + (emax - emin) * ii / nticks;
    }
    for (size_t x = 0; x < (size_t)nb * 9 * nticks; x++) results[x] = 0.0;
    for (int jj = 1; jj <= nb; jj++)
        for (int ii = 2; ii <= nptk; ii++) {
            double v[3], f[3], tmp[3][3];
            for (int d = 0; d < 3; d++) {
                v[d] = Vel(s, ii, jj, d);
                f[d] = F[((size_t)d * nptk + (ii - 1)) * nb + (jj - 1)];
            }
            for (int d1 = 0; d1 < 3; d1++)
                for (int d2 = 0; d2 < 3; d2++) tmp[d1][d2] = v[d1] * f[d2];
            double w = E(s, ii, jj);
            double fbe = 1.0 / (exp(FP4O_HBAR * w / FP4O_KB / s->T) - 1.0);
            double pre = fbe * (fbe + 1) * w;
            for (int d1 = 0; d1 < 3; d1++)
                for (int d2 = 0; d2 < 3; d2++) tmp[d1][d2] = pre * tmp[d1][d2];
            double lambda;
            if (omega_mode == 0) {
                double dot = 0.0;
                for (int d = 0; d < 3; d++) dot = dot + f[d] * v[d];
                lambda = dot / ((w + 1e-12) * nrm2_3(v));
            } else {
                lambda = w;
            }
            for (int k = 0; k < nticks; k++)
                if (ticks[k] > lambda)
                    for (int d1 = 0; d1 < 3; d1++)
                        for (int d2 = 0; d2 < 3; d2++) {
                            size_t o = (((size_t)k * 3 + d2) * 3 + d1) * nb + (jj - 1);
                            results[o] = results[o] + tmp[d1][d2];
                        }
        }
    double fac = (double)1e21f * (FP4O_HBAR * FP4O_HBAR);
    double den = FP4O_KB * s->T * s->T * V * nptk;
    for (size_t x = 0; x < (size_t)nb * 9 * nticks; x++) results[x] = fac * results[x] / den;
}

/* config.f90:503-518 symmetrize_tensor; crot(3,3,nsymm_rot) column-major. */
void fp4o_symmetrize_tensor(int nsymm_rot, const double *crot, double *t /* t(3,3) col-major */) {
    double acc[9] = {0};
    for (int is = 0; is < nsymm_rot; is++) {
        const double *R = crot + 9 * is;
        double m1[9];
        /* m1 = matmul(tensor, transpose(R)) */
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                double x = 0.0;
                for (int c = 0; c < 3; c++) x = x + t[a + 3 * c] * R[b + 3 * c];
                m1[a + 3 * b] = x;
            }
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                double x = 0.0;
                for (int c = 0; c < 3; c++) x = x + R[a + 3 * c] * m1[c + 3 * b];
                acc[a + 3 * b] = acc[a + 3 * b] + x;
            }
    }
    for (int x = 0; x < 9; x++) t[x] = acc[x] / nsymm_rot;
}

int fp4o_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
