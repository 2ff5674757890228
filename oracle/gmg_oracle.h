/*
 * gmg_oracle.h -- CPU FP64 restatement of the grid-mg-bench multigrid hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path
 * (tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py are
 * its only users).  Nothing in the product library links or calls it.
 *
 * Parity status: the reference (DanielRichtmann/grid-mg-bench) is a set of
 * header templates over the Grid library, which is not installed and cannot
 * be fetched, so the reference cannot be compiled here and ships no golden
 * vectors.  Every function below restates one reference function (cited by
 * file:line) and is pinned by the reference's own known-answer and identity
 * checks (geometry round trip, LUT consistency, Upstream == Dirsave links,
 * P R v = v, R P v_c = v_c, R D P = D_c, Im<v,Dc^+Dc v> = 0,
 * M = Mdiag + sum Mdir).  Absolute values of Grid's fine operator, its RNG
 * streams and its gauge generation are *parity unpinned*: the fine
 * Wilson-clover operator here is defined from its textbook form (DeGrand-
 * Rossi chiral gamma basis, the basis Grid uses) and inputs are generated by
 * this project, with the same bytes fed to the oracle and to the GPU.
 *
 * Conventions (all shared with the CUDA library):
 *   - lattice sites are lexicographic with x fastest: s = x + Lx*(y + Ly*(z + Lz*t))
 *   - complex numbers are interleaved (re, im) doubles
 *   - multi-RHS fields are [site][rhs][dof]   (the reference's 5-d layout with
 *     the RHS index fastest, CoarsenedMatrixUpstreamImprovedDirsaveLutMRHS.h:767-790)
 *   - basis ("subspace") is [i][site][dof]
 *   - coarse links are [point][site][row b][col bb] (Grid's A[p] lattice of
 *     row-major nbasis x nbasis matrices, CoarsenedMatrixUpstream.h:593)
 *   - stencil points: p<4 -> (dir p, +1), 4<=p<8 -> (dir p-4, -1), p=8 -> self
 */
#ifndef GMG_ORACLE_H
#define GMG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* geometry (GeometryRework.h:54-125) */
int  orc_point_from_dir_disp(int ndim, int dirs_faster, int dir, int disp);
void orc_geometry(int ndim, int dirs_faster, int* dirs, int* disps);
void orc_coarse_neighbors(const int* dims, int32_t* nbr);

/* coarsening lookup table (CoarseningLookupTableRework.h:114-179) */
int  orc_lut_populate(const int* fdims, const int* cdims, const int8_t* mask,
                      int32_t* lut, int32_t* sizes, int32_t* reverse);
void orc_outer_mask(const int* fdims, const int* cdims, int point, int8_t* mask);
void orc_block_parity_mask(const int* fdims, const int* cdims, int parity, int8_t* mask);

/* coarse stencil (CoarsenedMatrixUpstream.h:546-742) */
void orc_coarse_apply(const int* dims, int N, int R, const double* links,
                      const double* in, double* out, int op, int point, int hermitian);
void orc_coarse_apply_range(const int* dims, int N, int R, const double* links,
                            const double* in, double* out, int op, int point, int hermitian,
                            int64_t s0, int64_t s1);
void orc_coarse_g5(int64_t V, int N, int R, double* v);
/* OpenMP threads of the parallel loops (n <= 0: all); returns the previous count */
int  orc_set_threads(int n);

/* block projection / promotion / orthonormalisation
   (CoarsenedMatrixUpstreamImprovedDirsaveLut.h:70-240) */
void orc_block_project(const int* fdims, const int* cdims, int dof, int N, int R,
                       const double* basis, const double* fine, double* coarse,
                       const int8_t* mask);
void orc_block_promote(const int* fdims, const int* cdims, int dof, int N, int R,
                       const double* basis, const double* coarse, double* fine);
void orc_block_orthonormalise(const int* fdims, const int* cdims, int dof, int N,
                              double* basis, int passes);

/* chiral doubling (Benchmark_helpers.h:130-213) */
void orc_chiral_double(int64_t V, int dof, int nb, double* basis, double factor);
void orc_undo_chiral_double(int64_t V, int dof, int nb, double* basis);

/* fine Wilson-clover operator */
void orc_gamma(int mu, double* g);
void orc_clover_build(const int* dims, const double* U, double csw, double* clover);
void orc_wilson_clover_apply(const int* dims, const double* U, const double* clover,
                             double mass, int antiperiodic_t, int R,
                             const double* in, double* out, int op, int dir, int disp);

/* Galerkin coarse-operator construction
   (CoarsenedMatrixUpstream.h:755-931, ...DirsaveLut.h:927-1097, 1164-1196) */
void orc_coarsen_wilson(const int* fdims, const int* cdims, int N, const double* basis,
                        const double* U, const double* clover, double mass,
                        int antiperiodic_t, int hermitian, int variant, double* links);
void orc_coarsen_coarse(const int* fdims, const int* cdims, int Nf, int N,
                        const double* basis, const double* flinks, int fhermitian,
                        int hermitian, int variant, double* links);
void orc_construct_remaining_links(const int* dims, int N, double* links, int hermitian);

/* Rework 1/2/4-spin layout maps (Layout_converters.h:49-56,107-110) */
void orc_layout_vec_flat_to_spin(int64_t V, int N, int ncs, const double* in, double* out);
void orc_layout_link_flat_to_spin(int64_t V, int N, int ncs, const double* in, double* out);

/* red-black coarse operator (CoarsenedMatrixRework.h:178-245, 288-394, 617-679);
   half index h = x/2 + (Lx/2)*(y + Ly*(z + Lz*t)) on the sites of one parity */
void orc_pick_checkerboard(const int* dims, int cb, int64_t per_site, const double* full, double* half);
void orc_set_checkerboard(const int* dims, int cb, int64_t per_site, const double* half, double* full);
int  orc_invert_self_links(int64_t V, int N, const double* A8, double* Ainv);
void orc_coarse_rb_apply(const int* dims, int N, int R, const double* links, const double* self_inv,
                         int op, int cb, const double* in_half, double* out_half);
void orc_coarse_dhop(const int* dims, int N, int R, const double* links, int dag, const double* in, double* out);
void orc_coarse_mooee(const int* dims, int N, int R, const double* links, const double* self_inv, int op,
                      const double* in, double* out);

#ifdef __cplusplus
}
#endif
#endif
