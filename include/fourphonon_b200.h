/*
 * fourphonon_b200.h -- C-ABI of the B200 scattering-rate path.
 *
 * Each entry point replaces one Fortran subroutine of FourPhonon's hot path
 * and takes that subroutine's arguments in the same order, with the same
 * meaning, types and column-major layouts (indices stored in arrays are
 * 1-based, as in the reference).  The reference keeps the run parameters in
 * module globals (Src/config.f90:9-47); here they travel in fp4_globals.
 *
 * Array layouts (Fortran column-major):
 *   energy(nptk,nbands)             double, rad/ps
 *   velocity(nptk,nbands,3)         double, km/s
 *   eigenvect(nptk,nbands,nbands)   double complex (re,im interleaved)
 *   List(nlist), IJK(3,nptk)        int32
 *   Phi(3,3,3,Ntri), R_j(3,Ntri)    double (eV/A^3, nm), Index_*(Ntri) int32
 *   Psi(3,3,3,3,Ntri)               double (eV/A^4)
 *   rate(nbands,nlist)              double, THz
 *   N_plus(nlist*nbands) int32, N_plusplus(nlist*nbands) int64
 *
 * Every entry returns FP4_OK (0) or a negative FP4_E* code; the message of
 * the last failure on a context is returned by fp4_last_error().  Calls on
 * one context are not re-entrant (the reference calls them from the MPI main
 * thread); distinct contexts are independent.  All arrays are caller-owned
 * host memory; device copies are owned by the context.
 *
 * Limits: ngrid(d) <= 64, nbands <= 32, up to 8 temperatures in one call, and
 * for the four-phonon drivers 3*nlist*nptk < 2^31 - 2^20 work items (q, q',
 * channel); larger calls return FP4_E_ARG or FP4_E_CAPACITY.
 */
#ifndef FOURPHONON_B200_H
#define FOURPHONON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FP4_OK 0
#define FP4_E_ARG (-1)      /* bad shape / value / null pointer */
#define FP4_E_CUDA (-2)     /* CUDA runtime error (no device, launch failure...) */
#define FP4_E_CAPACITY (-3) /* a device work queue or table limit was exceeded */
#define FP4_E_TIMEOUT (-4)  /* a bounded device wait gave up */
#define FP4_E_STATE (-5)    /* call order (e.g. no system set) */

#define FP4_PREC_FP64 0  /* all-FP64 drop-in */
#define FP4_PREC_MIXED 1 /* split-bf16 tensor-core contraction (FP32 accumulate), FP64 filter/weights/reductions */
#define FP4_PREC_MIXED_SIMT 2 /* FP32 contraction on the CUDA cores, FP64 filter/weights/reductions */

typedef struct fp4_ctx fp4_ctx;

/* Run parameters held by module globals in the reference (config.f90:9-47). */
typedef struct {
    int32_t ngrid[3];     /* ngrid */
    int32_t nbands;       /* nbands = 3*natoms */
    double rlattvec[9];   /* rlattvec(3,3), column-major, nm^-1 */
    double T;             /* K */
    double scalebroad;    /* scalebroad */
    double omega_max;     /* omega_max (rad/ps) */
    int32_t onlyharmonic; /* logical onlyharmonic */
    int32_t nelements;    /* size of masses */
    int32_t natoms;       /* size of types */
    const double *masses; /* masses(nelements), amu */
    const int32_t *types; /* types(natoms), 1-based */
} fp4_globals;

/* Context on CUDA device `device` (-1: current device). */
int fp4_create(fp4_ctx **ctx, int device);
int fp4_destroy(fp4_ctx *ctx);
const char *fp4_last_error(const fp4_ctx *ctx);
/*
 * FP4_PREC_FP64 (default), FP4_PREC_MIXED or FP4_PREC_MIXED_SIMT for the rate
 * drivers.  FP4_PREC_MIXED runs the four-phonon RTA contraction on the tensor
 * cores (split bf16 operands, FP32 accumulation) when its tables fit in
 * shared memory, else as FP4_PREC_MIXED_SIMT; the other mixed drivers use
 * the FP32 CUDA-core contraction.  Filters, weights and sums stay FP64.
 */
int fp4_set_precision(fp4_ctx *ctx, int precision);

/*
 * Replaces NP_driver (Src/processes.f90:983-1067): per-mode counts of
 * allowed 3-phonon processes and their phase-space volumes.
 * Outputs N_plus(nlist*nbands), Pspace_plus_total(nbands,nlist), ...
 */
int fp4_np_driver(fp4_ctx *ctx, const fp4_globals *g, const double *energy, const double *velocity, int32_t nlist,
                  const int32_t *list, const int32_t *ijk, int32_t *n_plus, double *pspace_plus, int32_t *n_minus,
                  double *pspace_minus);

/* Replaces NP_driver_4ph (Src/processes.f90:2749-2847). */
int fp4_np_driver_4ph(fp4_ctx *ctx, const fp4_globals *g, const double *energy, const double *velocity,
                      int32_t nlist, const int32_t *list, const int32_t *ijk, int64_t *n_plusplus,
                      double *pspace_plusplus, int64_t *n_plusminus, double *pspace_plusminus, int64_t *n_minusminus,
                      double *pspace_minusminus);

/*
 * Replaces Ind_only_driver (Src/processes.f90:1198-1309): the 3-phonon index
 * lists Indof2ndPhonon_*(Ntotal), Indof3rdPhonon_*(Ntotal) in the
 * reference's order (per mode: j outer, q' inner, k innermost) at the Naccum
 * offsets of N_plus/N_minus (which the caller obtained from fp4_np_driver).
 */
int fp4_ind_only_driver(fp4_ctx *ctx, const fp4_globals *g, const double *energy, const double *velocity,
                        int32_t nlist, const int32_t *list, const int32_t *ijk, const int32_t *n_plus,
                        const int32_t *n_minus, int32_t *ind2_plus, int32_t *ind3_plus, int32_t *ind2_minus,
                        int32_t *ind3_minus);

/*
 * Replaces Ind_only_driver_4ph (Src/processes.f90:3080-3246): the 4-phonon
 * index lists (int64) in the reference's order (per mode: q', q'', j, k, l).
 * Sized by N_plusplus etc.; meant for grids whose lists fit in host memory.
 */
int fp4_ind_only_driver_4ph(fp4_ctx *ctx, const fp4_globals *g, const double *energy, const double *velocity,
                            int32_t nlist, const int32_t *list, const int32_t *ijk, const int64_t *n_plusplus,
                            const int64_t *n_plusminus, const int64_t *n_minusminus, int64_t *ind2_pp,
                            int64_t *ind3_pp, int64_t *ind4_pp, int64_t *ind2_pm, int64_t *ind3_pm,
                            int64_t *ind4_pm, int64_t *ind2_mm, int64_t *ind3_mm, int64_t *ind4_mm);

/*
 * Replaces RTA_driver (Src/processes.f90:1676-1775) and its GPU twin
 * RTA_driver_GPU_using_Ind (1778-1836): 3-phonon RTA rates at g->T.
 * rate_minus carries the driver's factor 1/2; rate = rate_plus + rate_minus.
 */
int fp4_rta_driver(fp4_ctx *ctx, const fp4_globals *g, const double *energy, const double *velocity,
                   const double *eigenvect, int32_t nlist, const int32_t *list, const int32_t *ijk, int32_t ntri,
                   const double *phi, const double *r_j, const double *r_k, const int32_t *index_i,
                   const int32_t *index_j, const int32_t *index_k, double *rate, double *rate_plus,
                   double *rate_minus, double *wp3_plus, double *wp3_minus);

/*
 * Replaces RTA_driver_4ph (Src/processes.f90:5174-5311) and its GPU twin
 * RTA_driver_4ph_GPU_using_Ind (5315-5387): 4-phonon RTA rates at g->T.
 * No index list is materialised: processes are enumerated, filtered and
 * contracted on the device.
 */
int fp4_rta_driver_4ph(fp4_ctx *ctx, const fp4_globals *g, const double *energy, const double *velocity,
                       const double *eigenvect, int32_t nlist, const int32_t *list, const int32_t *ijk, int32_t ntri,
                       const double *psi, const double *r_j, const double *r_k, const double *r_l,
                       const int32_t *index_i, const int32_t *index_j, const int32_t *index_k,
                       const int32_t *index_l, double *rate_4ph, double *rate_plusplus, double *rate_plusminus,
                       double *rate_minusminus, double *wp4_plusplus, double *wp4_plusminus, double *wp4_minusminus);

/*
 * Multi-temperature form of fp4_rta_driver_4ph: the matrix elements are
 * temperature independent, so they are contracted once and weighted for all
 * nT temperatures (the reference re-runs RTA_driver_4ph per temperature in
 * the loop of Src/ShengBTE.f90:787-1008).  g->T is ignored; outputs are
 * (nbands,nlist,nT).
 */
int fp4_rta_driver_4ph_multi_t(fp4_ctx *ctx, const fp4_globals *g, int32_t nT, const double *temperatures,
                               const double *energy, const double *velocity, const double *eigenvect, int32_t nlist,
                               const int32_t *list, const int32_t *ijk, int32_t ntri, const double *psi,
                               const double *r_j, const double *r_k, const double *r_l, const int32_t *index_i,
                               const int32_t *index_j, const int32_t *index_k, const int32_t *index_l,
                               double *rate_plusplus, double *rate_plusminus, double *rate_minusminus,
                               double *wp4_plusplus, double *wp4_plusminus, double *wp4_minusminus);

/*
 * Replaces Ind_driver (Src/processes.f90:524-707): per-process 3-phonon
 * scattering amplitudes Gamma_plus/Gamma_minus with their index lists in the
 * reference's order at the Naccum offsets of N_plus/N_minus, and the per-mode
 * rates (rate_minus with the factor 1/2, Gamma_minus without it).
 */
int fp4_ind_driver(fp4_ctx *ctx, const fp4_globals *g, const double *energy, const double *velocity,
                   const double *eigenvect, int32_t nlist, const int32_t *list, const int32_t *ijk,
                   const int32_t *n_plus, const int32_t *n_minus, int32_t ntri, const double *phi,
                   const double *r_j, const double *r_k, const int32_t *index_i, const int32_t *index_j,
                   const int32_t *index_k, int32_t *ind2_plus, int32_t *ind3_plus, double *gamma_plus,
                   int32_t *ind2_minus, int32_t *ind3_minus, double *gamma_minus, double *rate, double *rate_plus,
                   double *rate_minus, double *wp3_plus, double *wp3_minus);

/*
 * Replaces Ind_driver_4ph (Src/processes.f90:3551-3822) with Ind_plusplus,
 * Ind_plusminus and Ind_minusminus (3254-3548): the 4-phonon index lists of
 * the three channels in the reference's order at the Naccum offsets of
 * N_plusplus etc., each process's Gamma (hbarp^2 pi/8 WP4 |Vp|^2 in THz, no
 * extra factor), the per-mode rates (sum of the mode's Gammas), rate_4ph and
 * WP4 per mode.  Memory: 32 bytes per listed process on the device.
 */
int fp4_ind_driver_4ph(fp4_ctx *ctx, const fp4_globals *g, const double *energy, const double *velocity,
                       const double *eigenvect, int32_t nlist, const int32_t *list, const int32_t *ijk,
                       const int64_t *n_plusplus, const int64_t *n_plusminus, const int64_t *n_minusminus,
                       int32_t ntri, const double *psi, const double *r_j, const double *r_k, const double *r_l,
                       const int32_t *index_i, const int32_t *index_j, const int32_t *index_k,
                       const int32_t *index_l, int64_t *ind2_pp, int64_t *ind3_pp, int64_t *ind4_pp,
                       double *gamma_pp, int64_t *ind2_pm, int64_t *ind3_pm, int64_t *ind4_pm, double *gamma_pm,
                       int64_t *ind2_mm, int64_t *ind3_mm, int64_t *ind4_mm, double *gamma_mm, double *rate_4ph,
                       double *rate_plusplus, double *rate_plusminus, double *rate_minusminus,
                       double *wp4_plusplus, double *wp4_plusminus, double *wp4_minusminus);

/*
 * Replaces iteration0 (Src/iterations.f90:13-30).
 * allequilist(nsymm_rot,*) as ALLEquiList; F_n(nbands,nptk,3).
 */
int fp4_iteration0(fp4_ctx *ctx, const fp4_globals *g, int32_t nlist, const int32_t *nequi,
                   const int32_t *allequilist, int32_t nsymm_rot, const double *omega, const double *velocity,
                   const double *tau_zero, double *f_n);

/*
 * Replaces iteration (Src/iterations.f90:34-92): one Gauss-Seidel sweep of
 * the linearised BTE over the 3-phonon lists, F_n updated in place (same
 * sweep order), followed by no symmetrisation (the caller's loop applies it,
 * see fp4_symmetrize_fn).  id_equi(nsymm_rot,nptk) is symmetry_map's table
 * (Src/config.f90:397-419), symmetrizers(3,3,nptk).
 */
int fp4_iteration(fp4_ctx *ctx, const fp4_globals *g, int32_t nlist, const int32_t *nequi,
                  const int32_t *allequilist, const int32_t *typeofsymmetry, int32_t nsymm_rot,
                  const int32_t *id_equi, const double *symmetrizers, const int32_t *n_plus, const int32_t *n_minus,
                  int32_t ntotal_plus, int32_t ntotal_minus, const int32_t *ind2_plus, const int32_t *ind3_plus,
                  const int32_t *ind2_minus, const int32_t *ind3_minus, const double *omega,
                  const double *velocity, const double *gamma_plus, const double *gamma_minus,
                  const double *tau_zero, double *f_n);

/*
 * The Jacobi form of fp4_iteration (no counterpart in the reference, whose
 * update is Gauss-Seidel, Src/iterations.f90:34-92): same arguments and
 * layouts; every step of the sweep reads the F_n passed in and the new F_n
 * (with the site symmetrizers applied) is returned in f_n.  All steps run in
 * parallel on the device, so a sweep costs milliseconds where the in-order
 * sweep keeps one CTA busy; the iteration converges to the same kappa in more
 * sweeps.  Three-phonon processes only.
 */
int fp4_iteration_jacobi(fp4_ctx *ctx, const fp4_globals *g, int32_t nlist, const int32_t *nequi,
                         const int32_t *allequi, const int32_t *typeofsym, int32_t nsymm_rot, const int32_t *id_equi,
                         const double *symmetrizers, const int32_t *n_plus, const int32_t *n_minus,
                         int32_t ntotal_plus, int32_t ntotal_minus, const int32_t *ind2_plus, const int32_t *ind3_plus,
                         const int32_t *ind2_minus, const int32_t *ind3_minus, const double *energy,
                         const double *velocity, const double *gamma_plus, const double *gamma_minus,
                         const double *tau_zero, double *f_n);

/*
 * Replaces iteration_4ph (Src/iterations.f90:95-215): the sweep of
 * fp4_iteration with the ++, +- and -- lists of fp4_ind_driver_4ph added
 * (Gamma times F_l-F_j-F_k, F_l-F_j+F_k and F_l+F_j+F_k respectively).
 */
int fp4_iteration_4ph(fp4_ctx *ctx, const fp4_globals *g, int32_t nlist, const int32_t *nequi,
                      const int32_t *allequilist, const int32_t *typeofsymmetry, int32_t nsymm_rot,
                      const int32_t *id_equi, const double *symmetrizers, const int32_t *n_plus,
                      const int32_t *n_minus, int32_t ntotal_plus, int32_t ntotal_minus, const int64_t *n_plusplus,
                      const int64_t *n_plusminus, const int64_t *n_minusminus, int64_t ntotal_plusplus,
                      int64_t ntotal_plusminus, int64_t ntotal_minusminus, const int32_t *ind2_plus,
                      const int32_t *ind3_plus, const int32_t *ind2_minus, const int32_t *ind3_minus,
                      const int64_t *ind2_pp, const int64_t *ind3_pp, const int64_t *ind4_pp,
                      const int64_t *ind2_pm, const int64_t *ind3_pm, const int64_t *ind4_pm,
                      const int64_t *ind2_mm, const int64_t *ind3_mm, const int64_t *ind4_mm, const double *omega,
                      const double *velocity, const double *gamma_plus, const double *gamma_minus,
                      const double *gamma_pp, const double *gamma_pm, const double *gamma_mm,
                      const double *tau_zero, double *f_n);

/* F_n(:,q,:) symmetrisation of every q (Src/ShengBTE.f90:1288-1290). */
int fp4_symmetrize_fn(fp4_ctx *ctx, const fp4_globals *g, const double *symmetrizers, double *f_n);

/*
 * Replaces TConduct (Src/conductivity.f90:11-37).  V: unit-cell volume, nm^3.
 * thconductivity(nbands,3,3); thconductivitymode(nptk,nbands,3,3) may be NULL.
 */
int fp4_tconduct(fp4_ctx *ctx, const fp4_globals *g, double V, const double *omega, const double *velocity,
                 const double *f_n, double *thconductivity, double *thconductivitymode);

/*
 * Statistics of the last call on the context: surviving processes (all
 * channels), processes whose matrix element was contracted (the others have
 * a zero weight, w<=1.25 rad/ps), the device time of the whole call and of
 * its main rate kernel in milliseconds, and the number of kernel launches.
 * Any output pointer may be NULL.
 */
int fp4_last_stats(const fp4_ctx *ctx, int64_t *n_processes, int64_t *n_contracted, double *call_ms,
                   double *kernel_ms, int64_t *launches);

/*
 * Replace the sampled three-phonon drivers: NP_driver with
 * num_sample_process_3ph_phase_space > 0 (NP_plus_sample / NP_minus_sample,
 * Src/processes.f90:828-979) and RTA_driver with num_sample_process_3ph > 0
 * (RTA_plus_sample / RTA_minus_sample, 1474-1672, with the driver's x0.5 on the
 * emission rate): nsamples uniform draws of (q', j, k) per mode and channel,
 * scaled by nbands^2 nptk / nsamples.  The draws come from the same kind of
 * seeded stream as the four-phonon estimators (keys of their own).
 * nsamples < 2^32; nbands^2 nptk < 2^31.
 */
int fp4_np_driver_sample(fp4_ctx *ctx, const fp4_globals *g, const double *energy, const double *velocity,
                         int32_t nlist, const int32_t *list, const int32_t *ijk, int64_t nsamples, uint64_t seed,
                         int32_t *n_plus, double *pspace_plus, int32_t *n_minus, double *pspace_minus);
int fp4_rta_driver_sample(fp4_ctx *ctx, const fp4_globals *g, const double *energy, const double *velocity,
                          const double *eigenvect, int32_t nlist, const int32_t *list, const int32_t *ijk,
                          int32_t ntri, const double *phi, const double *r_j, const double *r_k,
                          const int32_t *index_i, const int32_t *index_j, const int32_t *index_k, int64_t nsamples,
                          uint64_t seed, double *rate, double *rate_plus, double *rate_minus, double *wp3_plus,
                          double *wp3_minus);

/*
 * Replace the sampled drivers: NP_driver_4ph with num_sample_process_4ph_phase_space
 * > 0 (NP_plusplus_sample etc., Src/processes.f90:2480-2746) and RTA_driver_4ph
 * with num_sample_process_4ph > 0 (RTA_plusplus_sample etc., 4811-5172):
 * nsamples uniform draws of (q', j, q'', k, l) per mode and channel, scaled by
 * nbands^3 nptk^2 / nsamples.  The reference draws from an unseeded
 * random_number; here the draws come from a counter-based splitmix64 stream
 * keyed by (seed, mode, channel, sample), so a (seed, nsamples) pair always
 * gives the same estimate.  nsamples < 2^32.  The multi-temperature form
 * weights the same samples for nT temperatures (outputs (nbands,nlist,nT)).
 */
int fp4_np_driver_4ph_sample(fp4_ctx *ctx, const fp4_globals *g, const double *energy, const double *velocity,
                             int32_t nlist, const int32_t *list, const int32_t *ijk, int64_t nsamples,
                             uint64_t seed, int64_t *n_plusplus, double *pspace_plusplus, int64_t *n_plusminus,
                             double *pspace_plusminus, int64_t *n_minusminus, double *pspace_minusminus);
int fp4_rta_driver_4ph_sample(fp4_ctx *ctx, const fp4_globals *g, const double *energy, const double *velocity,
                              const double *eigenvect, int32_t nlist, const int32_t *list, const int32_t *ijk,
                              int32_t ntri, const double *psi, const double *r_j, const double *r_k,
                              const double *r_l, const int32_t *index_i, const int32_t *index_j,
                              const int32_t *index_k, const int32_t *index_l, int64_t nsamples, uint64_t seed,
                              double *rate_4ph, double *rate_plusplus, double *rate_plusminus,
                              double *rate_minusminus, double *wp4_plusplus, double *wp4_plusminus,
                              double *wp4_minusminus);
int fp4_rta_driver_4ph_sample_multi_t(fp4_ctx *ctx, const fp4_globals *g, int32_t nT, const double *temperatures,
                                      const double *energy, const double *velocity, const double *eigenvect,
                                      int32_t nlist, const int32_t *list, const int32_t *ijk, int32_t ntri,
                                      const double *psi, const double *r_j, const double *r_k, const double *r_l,
                                      const int32_t *index_i, const int32_t *index_j, const int32_t *index_k,
                                      const int32_t *index_l, int64_t nsamples, uint64_t seed,
                                      double *rate_plusplus, double *rate_plusminus, double *rate_minusminus,
                                      double *wp4_plusplus, double *wp4_plusminus, double *wp4_minusminus);

/*
 * Replace CumulativeTConduct (Src/conductivity.f90:64-97) and
 * CumulativeTConductOmega (100-148): ticks(nticks) (mean free paths in nm,
 * 10**(8(i-1)/(nticks-1)-2) in default REAL; or angular frequencies
 * emin+(emax-emin)*i/nticks with emax*1.1) and results(nbands,3,3,nticks),
 * the kappa of the modes whose mean free path (omega) lies below each tick.
 * The reference's nticks is 100 (config.f90:133).
 */
int fp4_cumulative_tconduct(fp4_ctx *ctx, const fp4_globals *g, double V, const double *omega,
                            const double *velocity, const double *f_n, int32_t nticks, double *ticks,
                            double *results);
int fp4_cumulative_tconduct_omega(fp4_ctx *ctx, const fp4_globals *g, double V, const double *omega,
                                  const double *velocity, const double *f_n, int32_t nticks, double *ticks,
                                  double *results);

/*
 * Replace eigenDM (Src/phonon_routines.f90:12-81) with phonon_phonopy
 * (84-307) for a Phonopy FORCE_CONSTANTS_2ND without the dielectric
 * correction when nonanalytic is set (lines 158-247): omega(nptk,nbands),
 * velocity(nptk,nbands,3) and eigenvect(nptk,nbands,nbands) (complex,
 * interleaved) on the Gamma-centred grid of g. lattvec(3,3) is in nm,
 * cartesian(3,natoms) in nm, scell the supercell,
 * fc(natoms,3,scell(1),scell(2),scell(3),natoms,3) the mass-reduced force
 * constants of read2fc (Src/input.f90:18-79), epsilon(3,3) and
 * born(3,3,natoms) the dielectric tensor and Born charges of CONTROL, V the
 * cell volume in nm^3 and symmetrizers(3,3,nptk) those of symmetry_map.
 * g->rlattvec gives the grid, g->masses and g->types the mass products.
 * Eigenvectors carry LAPACK's freedom: an arbitrary phase per branch and an
 * arbitrary basis inside a degenerate set.
 */
int fp4_eigen_dm(fp4_ctx *ctx, const fp4_globals *g, const double *lattvec, const double *cartesian,
                 const int32_t scell[3], const double *fc, int32_t nonanalytic, const double *epsilon,
                 const double *born, double V, const double *symmetrizers, double *omega, double *velocity,
                 double *eigenvect);

/*
 * Allocation-free form of fp4_np_driver_4ph, for callers that cannot
 * allocate device memory (a host whose device memory all comes from its own
 * pool, or code embedded in a process whose allocator it must not touch).
 * It has no counterpart in the reference.
 *
 * Same counts and phase spaces as fp4_np_driver_4ph, but: no context; every
 * array argument is a DEVICE pointer (energy(nptk,nbands),
 * velocity(nptk,nbands,3), List(nlist) in, the six per-mode outputs out);
 * `stream` is a cudaStream_t (NULL: the default stream), synchronised before
 * the call returns.  Scratch lives in one fixed 12 MiB (12,582,912 B) device
 * array that the library holds on every GPU it is loaded on until the process
 * exits.  A call needs nptk*nbands*32 + nptk*4 + nlist*4 + nlist*nbands*48
 * bytes plus 256 B of counters, each of the five parts rounded up to 256 B:
 * e.g. a 24^3 grid with 12 branches fits when List is an irreducible wedge
 * (nlist up to about 8,000 points) but not the full grid.  Larger calls, and
 * calls with more than 2^31 - 2^20 work items (3*nlist*nptk), return
 * FP4_E_CAPACITY before any device work; a List entry outside
 * [1, nptk] returns FP4_E_ARG.  The first call in each CUDA context looks up
 * the array's device address in that context, so make that call before any
 * stream capture.  All calls share the array: calls that
 * overlap on the GPU (other threads, other streams) race and must be
 * serialised by the caller.  No cudaMalloc/cudaFree is ever called.
 */
int fp4_np_driver_4ph_noalloc(const fp4_globals *g, const double *energy, const double *velocity, int32_t nlist,
                              const int32_t *list, int64_t *n_plusplus, double *pspace_plusplus, int64_t *n_plusminus,
                              double *pspace_plusminus, int64_t *n_minusminus, double *pspace_minusminus,
                              void *stream);

/*
 * Inspection of the last four-phonon RTA call (fp4_rta_driver_4ph[_multi_t]):
 * for irreducible point ll (0-based) and temperature index t, the rates and
 * WP4 of each branch (nbands values per output) from the processes whose
 * second phonon q' lies in [ii0, ii1) (0-based grid indices), normalised as
 * the full driver normalises them.  Over a partition of the grid these sum to
 * the driver's outputs.  No counterpart in the reference: it lets a large
 * grid be checked against a CPU restatement of a few q' points.
 */
int fp4_rta4_partials(fp4_ctx *ctx, int32_t ll, int32_t ii0, int32_t ii1, int32_t t, double *rate_pp,
                      double *rate_pm, double *rate_mm, double *wp_pp, double *wp_pm, double *wp_mm);

/*
 * Self-check of the tensor-core path (no counterpart in the reference): on
 * the current device, D(128,N) = A(128,K) * B(N,K)^T with bf16 A and B
 * (row-major host arrays of raw bf16 bits) and FP32 accumulation, through the
 * same shared-memory layout, tcgen05.mma, mbarrier and TMEM read-back that the
 * mixed-precision four-phonon contraction uses.  K a multiple of 16 up to
 * 1024, N a multiple of 16 in [16, 256]; D is a row-major host array.
 */
int fp4_tc_selftest(int32_t K, int32_t N, const uint16_t *A, const uint16_t *B, float *D);

/*
 * Work counters of the last four-phonon call: [0] surviving processes,
 * [1] contracted processes, [2] broadening evaluations (one per (q'',k,l)
 * candidate triple), [3] energy tests in the sorted windows, [4] reciprocal
 * cluster tables built on the CUDA cores (one per branch i, or per work item
 * when all branches are built at once), [5] (i,j) tables built for the
 * tensor cores, [6] tensor-core work in units of one 128 x 16 x 16 product
 * (a tcgen05.mma K-step of N columns counts N/16; 65,536 flops per unit),
 * [7] 1 if the contraction ran on the tensor cores, else 0.
 */
int fp4_last_counters(const fp4_ctx *ctx, int64_t counters[8]);

/*
 * Where the last four-phonon work kernel spent its time, in SM clock cycles
 * summed over its CTAs: [0] whole work items, [1] the contraction and
 * weighting of the queued processes (phase B) within them ([0] - [1] is the
 * enumeration and energy filter, phase A).  Tensor-core contraction only,
 * summed over the CTAs' threads that time them: [2] building the reciprocal
 * cluster and B tables, and per chunk of 128 processes, summed over the two
 * warpgroups: [3] gathering the A rows, [4] the product and the weights up
 * to the end of the wait, [5] the epilogue; [6..7] reserved (0).  Not part of
 * the reference.
 */
int fp4_last_phase_cycles(const fp4_ctx *ctx, int64_t cycles[8]);

/*
 * Run the context's work on an existing CUDA stream (a cudaStream_t passed
 * as void*); NULL restores the context's own stream.  Not part of the
 * reference interface: lets a host that owns a stream order these calls
 * with its own work.
 */
int fp4_set_stream(fp4_ctx *ctx, void *stream);

/*
 * Device copies of unchanged inputs are reused between calls (enable=1,
 * default); enable=0 copies every input on every call.
 */
int fp4_set_upload_cache(fp4_ctx *ctx, int enable);

/*
 * Serving: many 3ph+4ph RTA solves resident on one GPU.  No counterpart in
 * the reference, which runs one solve per process.
 *
 * fp4_server_create reserves the work queues (sized for max_bands branches)
 * and captures the tick graph.  On failure *srv may still hold a server whose
 * fp4_server_last_error explains the failure; destroy it.  hbm_budget_bytes
 * bounds the queues plus the footprints of the admitted solves.
 *
 * fp4_server_admit uploads one solve into a free slot: the arrays of
 * fp4_rta_driver (3ph) and fp4_rta_driver_4ph (4ph), at g->T, plus the
 * wedge's Nequi, ALLEquiList(nsymm_rot,nlist), crotations(3,3,nsymm_rot) and
 * the cell volume (nm^3) for kappa.  It returns FP4_E_STATE when no slot is
 * free or the budget is in use (retry after a collect), FP4_E_CAPACITY when
 * the solve can never fit.
 *
 * fp4_server_tick runs up to max_items work items (q, q', channel), shared
 * equally among the running solves, in one launch of the multi-solve kernel,
 * finishes the solves whose work is complete (rates, tau, iteration0,
 * TConduct, symmetrised kappa) and lists their slots in finished[] (room for
 * max_slots entries).  It returns when the tick has run.
 *
 * fp4_server_collect copies a finished slot's results (each pointer may be
 * NULL): rate_plus/rate_minus (3ph; minus with the factor 1/2), the three 4ph
 * rates (nbands*nlist each), kappa per branch (nbands x 3x3, column-major
 * blocks), kappa (3x3) and the number of surviving 3ph+4ph processes, then
 * frees the slot.
 */
typedef struct fp4_server fp4_server;
int fp4_server_create(fp4_server **srv, int device, int precision, int32_t max_slots, int32_t max_bands,
                      int64_t hbm_budget_bytes);
int fp4_server_destroy(fp4_server *srv);
const char *fp4_server_last_error(const fp4_server *srv);
int64_t fp4_server_footprint(int32_t nbands, int32_t nlist, const int32_t ngrid[3], int32_t ntri3, int32_t ntri4,
                             int32_t nsymm_rot);
int fp4_server_admit(fp4_server *srv, const fp4_globals *g, const double *energy, const double *velocity,
                     const double *eigenvect, int32_t nlist, const int32_t *list, const int32_t *ijk, int32_t ntri3,
                     const double *phi, const double *r_j3, const double *r_k3, const int32_t *index_i3,
                     const int32_t *index_j3, const int32_t *index_k3, int32_t ntri4, const double *psi,
                     const double *r_j4, const double *r_k4, const double *r_l4, const int32_t *index_i4,
                     const int32_t *index_j4, const int32_t *index_k4, const int32_t *index_l4, int32_t nsymm_rot,
                     const int32_t *nequi, const int32_t *allequilist, const double *crotations, double volume,
                     int32_t *slot);
int fp4_server_tick(fp4_server *srv, int64_t max_items, int32_t *finished, int32_t *nfinished);
int fp4_server_collect(fp4_server *srv, int32_t slot, double *rate3_plus, double *rate3_minus, double *rate4_pp,
                       double *rate4_pm, double *rate4_mm, double *kappa_branch, double *kappa,
                       int64_t *n_processes);
int fp4_server_status(const fp4_server *srv, int32_t *running, int32_t *done, int64_t *bytes_in_use,
                      double *last_tick_ms, int64_t *ticks);

#ifdef __cplusplus
}
#endif
#endif
