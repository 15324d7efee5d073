/*
 * pd_oracle.h -- CPU FP64 restatement of PeriDyn's per-step force path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA library is
 * compared against; it is never linked into, loaded by, or called from the
 * product library.  Only tests/, __graft_entry__.smoke() and the cpu_baseline
 * / reference arm of bench.py may load it.
 *
 * Every routine restates one function of the reference (PeriDyn v0.2.0,
 * Julia) literally, in the reference's loop order and floating-point
 * expression order, compiled with -ffp-contract=off so that no multiply-add
 * is fused (Julia fuses nothing outside muladd/@fastmath).
 *
 * Layouts are the reference's own: 3xN column-major Float64 for positions,
 * velocities and accelerations; family is M'xN column-major Int64, 1-based,
 * 0 = padding, each column in DESCENDING index order; intact is M'xN Bool.
 *
 * Parity status: the reference ships no tests, fixtures or golden vectors,
 * and Julia is not installed here, so this restatement cannot be checked
 * against reference outputs ("parity unpinned" by the reference itself).  It
 * is pinned instead by analytical known-answer tests derived from the
 * reference formulas (homogeneous stretch, conservation, rigid motion,
 * lattice neighbour counts) in tests/test_oracle_known_answers.py.
 */
#ifndef PD_ORACLE_H
#define PD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Julia fld(x, y) for Float64: round((x - mod(x, y)) / y).  */
double or_fld(double x, double y);
/* Julia Float64^Float64 for the exponents the contact law uses: the
 * compensated integer power of base/math.jl (pow_body) when y is integral,
 * libm pow otherwise. */
double or_pow(double x, double y);

/* peri.jl:533-576 cal_family!/cal_family + general_material.jl:85-90
 * (trim + reverse).  x: 3xn.  family_out: capacity max_neigh' x n where
 * max_neigh' = min(max_neigh, n).  On success *rows_out = M' and the first
 * M'*n entries of family_out hold the trimmed, reversed family (column-major,
 * leading dimension M').  Returns 0, or 3 when a family does not fit
 * (the reference raises a BoundsError there). */
int or_cal_family(int64_t n, const double *x, double horizon, int64_t max_neigh,
                  int64_t *family_out, int64_t *rows_out);

/* peri.jl:342-354 weighted_volume. */
void or_weighted_volume(int64_t n, const double *x, const double *vol,
                        int64_t M, const int64_t *family, double *m);

/* peri.jl:155-172 dilatation! (CPU). nthreads>1 runs the i-loop in parallel
 * (each theta[i] is owned by one thread, so the result is identical). */
void or_dilatation(int64_t n, const double *y, const double *x,
                   const uint8_t *intact, const int64_t *family, int64_t M,
                   const double *vol, const double *m, double *theta,
                   int nthreads);

/* general_material.jl:296-369 force_density_T! (CPU) with the bond laws of
 * bond_based.jl:225-231 (kind 0) and ordinary_state_based.jl:176-187
 * (kind 1).  f,y: 3xn block slices; type_rel: 1-based type within the
 * block; cs/c/K/G: ntypes x ntypes column-major; density: ntypes.
 * nthreads==1 reproduces the serial summation order exactly; nthreads>1
 * mirrors Threads.@threads with atomic scatter (order-dependent rounding). */
void or_force_density_T(int kind, int64_t n, int64_t M, double *f,
                        const double *y, const double *x,
                        const int64_t *family, uint8_t *intact,
                        const int64_t *type_rel, int64_t ntypes,
                        const double *cs, const double *density,
                        const double *vol, const double *c,
                        const double *m, const double *theta,
                        const double *K, const double *G, int nthreads);

/* Elasto-plastic solid (elasto_plastic.jl), single-threaded.
 * or_td_norm2: peri.jl:411-445 loop_over_neighs! with td_norm2_ij!
 *   (elasto_plastic.jl:274-288): td_norm2[i] = sum over intact bonds of
 *   td^2 V_j; bonds with s >= cs are cleared (as that loop does).
 * or_force_density_ep: general_material.jl:296-369 with
 *   force_density_t_ij (elasto_plastic.jl:215-242); edp (M x n) is updated
 *   in place.  psi: ntypes x ntypes yield values (init, :60-68). */
void or_td_norm2(int64_t n, int64_t M, const double *y, const double *x, const int64_t *family,
                 uint8_t *intact, const int64_t *type_rel, int64_t ntypes, const double *cs,
                 const double *vol, const double *m, const double *theta, const double *G,
                 const double *edp, double *td_norm2);
void or_force_density_ep(int64_t n, int64_t M, double *f, const double *y, const double *x,
                         const int64_t *family, uint8_t *intact, const int64_t *type_rel, int64_t ntypes,
                         const double *cs, const double *density, const double *vol, const double *m,
                         const double *theta, const double *K, const double *G, const double *psi,
                         const double *td_norm2, double *edp);

/* general_material.jl:243-255: the "deformed" gate.  Returns 1 when
 * isapprox(y .- y[:,1] .+ x[:,1], x) holds (rigid translate; skip forces). */
int or_isapprox_rigid(int64_t n, const double *y, const double *x);

/* contacts.jl:403-476 update_contact_neighs! (ContactModel12).  x11: 3xn1
 * positions of the particles of pair[1], x22: 3xn2 of pair[2].  neighs:
 * rows x n1 column-major (rows = RM.max_neighs). */
void or_contact12_neighs(int64_t n1, const double *x11, int64_t n2,
                         const double *x22, double distance, int64_t rows,
                         int64_t *neighs);

/* contacts.jl:210-247 short_range_contact! (ContactModel12, CPU) with the
 * force law of nonlinearspring.jl:124-145. */
void or_contact12_force(int64_t n1, int64_t rows, const int64_t *neighs,
                        const double *x1, const double *x2, double *f1,
                        double *f2, const double *vol1, const double *vol2,
                        const double *den1, const double *den2,
                        double equi_dist, double exponent, double stiffness);

/* peri.jl:500-520 get_cells + contacts.jl:539-573 / 591-605
 * update_contact_neighs! (ContactModel11, CPU, literal merge walk). */
void or_contact11_neighs(int64_t n, const double *x, int64_t M,
                         const int64_t *family, const uint8_t *intact,
                         double search_distance, double equi_dist,
                         int64_t max_part, int64_t rows, int64_t *neighbors);

/* Ordered variant of contacts.jl:539-573: every broken-bond family member
 * in an adjacent cell and within equi_dist, in family order, up to rows. */
void or_contact11_neighs_ordered(int64_t n, const double *x, int64_t M,
                                 const int64_t *family, const uint8_t *intact,
                                 double search_distance, double equi_dist,
                                 int64_t max_part, int64_t rows, int64_t *neighbors);

/* contacts.jl:357-381 short_range_contact! (ContactModel11, CPU). */
void or_contact11_force(int64_t n, int64_t rows, const int64_t *neighs,
                        const double *x1, double *f1, const double *vol1,
                        const double *den1, double equi_dist, double exponent,
                        double stiffness);

#ifdef __cplusplus
}
#endif
#endif
