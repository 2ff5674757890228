/*
 * gmg.h -- C ABI of the B200-native multigrid hot path (libgmg_b200.so).
 *
 * Drop-in boundary for grid-mg-bench's coarse-operator and aggregation
 * classes.  Every entry point names the reference interface it replaces
 * (paths inside DanielRichtmann/grid-mg-bench).  Plain pointers and sizes
 * only; streams are cudaStream_t values passed as `gmg_stream` (NULL = the
 * legacy default stream).  All calls are stream-ordered and asynchronous
 * unless stated; calls on one handle are not thread-safe, calls on different
 * handles are.  Every call returns a gmg_status; gmg_last_error() gives the
 * message of the last failure on the calling thread.
 *
 * Layouts (complex numbers interleaved re, im; sites lexicographic, x fastest):
 *   fine field       [site][rhs][dof]          dof = 12 (spin-major, colour fastest)
 *   coarse field     [site][rhs][nbasis]       (the reference's 5-d MRHS layout,
 *                                               ...LutMRHS.h:767-790, RHS fastest)
 *   basis            [i][site][dof]            (Aggregation::subspace)
 *   coarse links     [point][site][b][bb]      (CoarsenedMatrix::A, row-major N x N)
 *   gauge field      [site][mu][3][3]
 *   stencil points   p<4: (dir p, +1); 4<=p<8: (dir p-4, -1); p=8: self
 *                    (GeometryRework.h:54-125, directions-faster order)
 */
#ifndef GMG_H
#define GMG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* gmg_stream;

typedef enum {
  GMG_OK = 0,
  GMG_ERR_ARGUMENT = 1,      /* null pointer / out-of-range argument */
  GMG_ERR_SHAPE = 2,         /* non-conformable sizes (Grid's conformable() abort) */
  GMG_ERR_STATE = 3,         /* handle not ready (links / basis / gauge not set) */
  GMG_ERR_CUDA = 4,          /* CUDA runtime error */
  GMG_ERR_NOMEM = 5,         /* device allocation failed */
  GMG_ERR_UNSUPPORTED = 6,   /* precision / size combination not built */
  GMG_ERR_NONFINITE = 7,     /* NaN or Inf detected */
  GMG_ERR_NOT_CONVERGED = 8, /* iterative solve hit its iteration limit */
  GMG_ERR_TIMEOUT = 9        /* a bounded device wait ran out */
} gmg_status;

typedef enum { GMG_F64 = 0, GMG_F32 = 1, GMG_BF16 = 2, GMG_F16 = 3 } gmg_prec;

typedef enum { GMG_OP_M = 0, GMG_OP_MDAG = 1, GMG_OP_MDIAG = 2, GMG_OP_MDIR = 3 } gmg_op;

const char* gmg_last_error(void);
const char* gmg_version(void);

/* ------------------------------------------------------------------------ */
/* Geometry and lookup tables                                                */
/* ------------------------------------------------------------------------ */

/* Rework::Geometry::PointFromDirDisp (GeometryRework.h:65-98); -1 on bad input. */
int gmg_point_from_dir_disp(int ndim, int dirs_faster, int dir, int disp);

/* CoarseningLookupTable::populate (CoarseningLookupTableRework.h:114-179) for
   mask_kind: -1 = full block, 0..7 = outer face of stencil point p
   (CoarsenedMatrixUpstream.h:815-821), 9 = even blocks, 10 = odd blocks.
   Host outputs: lut[Vc][bv] (-1 padded), sizes[Vc], reverse[Vf] (nullable). */
gmg_status gmg_lut_build(const int fine_dims[4], const int coarse_dims[4], int mask_kind,
                         int32_t* lut, int32_t* sizes, int32_t* reverse);

/* ------------------------------------------------------------------------ */
/* Coarse stencil -- CoarsenedMatrix (CoarsenedMatrixUpstream.h:515-753)    */
/* ------------------------------------------------------------------------ */
typedef struct gmg_coarse gmg_coarse;

/* CoarsenedMatrix(GridCartesian& CoarseGrid, int hermitian) (CoarsenedMatrixUpstream.h:745-753) */
gmg_status gmg_coarse_create(const int dims[4], int nbasis, int hermitian, gmg_coarse** h);
gmg_status gmg_coarse_destroy(gmg_coarse* h);

/* Write / read the public link fields A[p] (CoarsenedMatrixUpstream.h:536, written
   by the benchmarks at Benchmark_coarse_operator.cc:121-127).  `links` is
   [9][V][N][N] complex128 on the host (on_device=0) or the device (1).
   Setting links refreshes every reduced-precision copy already prepared. */
gmg_status gmg_coarse_set_links(gmg_coarse* h, const double* links, int on_device, gmg_stream s);
gmg_status gmg_coarse_get_links(gmg_coarse* h, double* links, int on_device, gmg_stream s);

/* Build the link copy used by `compute` (F32, BF16 or F16); F64 needs none. */
gmg_status gmg_coarse_prepare(gmg_coarse* h, gmg_prec compute, gmg_stream s);

/* M / Mdag / Mdiag / Mdir(point) on nrhs right-hand sides
   (CoarsenedMatrixUpstream.h:546-742; multi-RHS ...LutMRHS.h:736-947).
   in, out: device coarse fields [V][nrhs][N] of type vec_prec (F64 or F32).
   compute: F64 (FP64 links+vectors), F32 (FP32), BF16 / F16 (tensor cores,
   FP32 accumulation, FP32 vectors).  Mdag is G5C M G5C unless hermitian,
   fused into the load/store.  active (device int32[n_active], nullable)
   restricts the apply to those RHS slots; other slots of `out` are untouched. */
gmg_status gmg_coarse_apply(gmg_coarse* h, gmg_op op, int point, gmg_prec compute,
                            gmg_prec vec_prec, int nrhs, const void* in, void* out,
                            const int32_t* active, int n_active, gmg_stream s);

/* The launch shape the autotuner chose for the tensor-core stencil of this
   handle: CTAs per SM and stencil points per stage, for an apply of nrhs
   right-hand sides over npoints stencil points (9 for M) in `compute`
   (GMG_BF16 / GMG_F16); 0, 0 before the first such apply.  The first apply
   of each (nbasis, padded nrhs, volume, point count, operand kind) times every
   shape that fits and keeps the fastest, each timed launch after a write of a
   192 MB buffer that evicts L2 (as a solve's other work does); that buffer is
   allocated on the first tuning call on a device and kept for the process.
   No counterpart in the reference. */
gmg_status gmg_coarse_tuned_shape(gmg_coarse* h, int nrhs, int npoints, gmg_prec compute, int* ctas,
                                  int* points_per_stage);
/* Force the tensor-core stencil shape of this handle (CTAs per SM 1 or 2,
   points per stage 1-4); 0, 0 restores autotuning.  A forced shape that does
   not fit a call (the point count not a multiple of it, TMEM or shared memory
   too small) falls back to the tuned one.  No counterpart in the reference. */
gmg_status gmg_coarse_set_shape(gmg_coarse* h, int ctas, int points_per_stage);
/* Allocation-free form of gmg_coarse_apply for the BF16 / F16 tensor-core
   path (no counterpart in the reference).  For callers that cannot let the
   library allocate while they run -- a solver loop that must not stall the
   device (cudaMalloc / cudaFree may synchronise) or an application whose
   device memory all comes from its own pool allocator.  The packed
   right-hand sides go to a fixed 16 MiB array of device memory that every
   GPU loading the library holds until exit; requests needing more (V * Kc *
   2 * ceil16(R) * 16 bytes, Kc = ceil16(nbasis)/8) return
   GMG_ERR_UNSUPPORTED.  Vectors are FP32 [V][nrhs][N]; gmg_coarse_prepare
   (which allocates) must have run for `compute` first.  Every call looks up
   the array's device address on the current device (cudaGetSymbolAddress),
   which allocates nothing once the library's device code is loaded; with
   lazy module loading (the CUDA default) the first call on a device may load
   it and so commit the 16 MiB at that moment.  A caller that must not
   allocate mid-run makes one warm-up call at setup, before any stream
   capture.  All calls share the array: calls that overlap on the GPU race
   and must be serialised by the caller. */
gmg_status gmg_coarse_apply_noalloc(gmg_coarse* h, gmg_op op, int point, gmg_prec compute, int nrhs,
                                    const float* in, float* out, const int32_t* active, int n_active,
                                    gmg_stream s);

/* MdirAll (CoarsenedMatrixUpstream.h:700-713): out8[p] = A_p in(nbr_p), p < 8. */
gmg_status gmg_coarse_mdir_all(gmg_coarse* h, gmg_prec compute, gmg_prec vec_prec, int nrhs,
                               const void* in, void* const* out8, gmg_stream s);

/* ConstructRemainingLinks / ForceHermitian (...DirsaveLut.h:1164-1196,
   CoarsenedMatrixUpstream.h:956-976): rebuild the 4 forward links from the
   backward ones, A_{+mu}(x) = S o A_{-mu}(x+mu)^dag (S = 1 if hermitian). */
gmg_status gmg_coarse_construct_remaining_links(gmg_coarse* h, gmg_stream s);

/* ------------------------------------------------------------------------ */
/* Red-black (checkerboarded) coarse operator: the Schur interface of        */
/* Rework::CoarsenedMatrix (CoarsenedMatrixRework.h:178-245, 288-394,        */
/* 617-679).  A half field holds the sites of one parity q = (x+y+z+t) % 2    */
/* as [V/2][nrhs][nbasis], half index h = x/2 + (Lx/2)*(y + Ly*(z + Lz*t))    */
/* (Grid's red-black grid, checkerboarded in x); all extents must be even.   */
/* ------------------------------------------------------------------------ */
typedef enum {
  GMG_RB_MEOOE = 0,         /* out (parity 1-cb) = sum of the 8 hops of in (parity cb): DhopOE / DhopEO */
  GMG_RB_MEOOE_DAG = 1,     /* G5C Meooe G5C (DhopInternal with dag, :289-346) */
  GMG_RB_MOOEE = 2,         /* out (parity cb) = A_self in                 (Mooee, :202) */
  GMG_RB_MOOEE_DAG = 3,     /* adj(A_self) in                              (MooeeDag, :206) */
  GMG_RB_MOOEE_INV = 4,     /* A_self^-1 in, after gmg_coarse_invert_self  (MooeeInv, :204) */
  GMG_RB_MOOEE_INV_DAG = 5  /* adj(A_self^-1) in                           (MooeeInvDag, :208) */
} gmg_rb_op;

/* InvertSelfStencilPoint (CoarsenedMatrixRework.h:642-668): inverse of every
   site's self-stencil link, on the device in FP64 (Gauss-Jordan, partial
   pivoting), kept with an FP32 copy.  Synchronises the stream; returns
   GMG_ERR_NONFINITE if a self link is singular.  Setting or rebuilding the
   links drops the inverse. */
gmg_status gmg_coarse_invert_self(gmg_coarse* h, gmg_stream s);

/* Meooe / MeooeDag on half fields (in of parity cb, out of parity 1-cb) and
   Mooee / MooeeDag / MooeeInv / MooeeInvDag (in and out of parity cb).
   compute as for gmg_coarse_apply: the BF16 / F16 hops run on the tensor
   cores (F32 vectors); the self-point ops run in FP32 for those requests. */
gmg_status gmg_coarse_apply_rb(gmg_coarse* h, gmg_rb_op op, int cb, gmg_prec compute, gmg_prec vec_prec,
                               int nrhs, const void* in, void* out, gmg_stream s);

/* Dhop (CoarsenedMatrixRework.h:210-217) on the full grid: the 8 hopping
   points; dag != 0 gives G5C Dhop G5C. */
gmg_status gmg_coarse_dhop(gmg_coarse* h, int dag, gmg_prec compute, gmg_prec vec_prec, int nrhs,
                           const void* in, void* out, gmg_stream s);

/* Mooee family on the full grid (op GMG_RB_MOOEE .. GMG_RB_MOOEE_INV_DAG). */
gmg_status gmg_coarse_mooee(gmg_coarse* h, gmg_rb_op op, gmg_prec compute, gmg_prec vec_prec, int nrhs,
                            const void* in, void* out, gmg_stream s);

/* Grid's pickCheckerboard / setCheckerboard on device fields [V][per_site]
   complex (F64 or F32): full -> half of parity cb, and half -> those sites of full. */
gmg_status gmg_pick_checkerboard(const int dims[4], int cb, int per_site, gmg_prec prec, const void* full,
                                 void* half, gmg_stream s);
gmg_status gmg_set_checkerboard(const int dims[4], int cb, int per_site, gmg_prec prec, const void* half,
                                void* full, gmg_stream s);

/* Error code recorded on the device by this handle's tensor-core kernels
   (0 = none; otherwise a bounded wait ran out and the kernel returned early),
   read after a device synchronisation and then cleared.  Returns
   GMG_ERR_TIMEOUT when *code != 0.  No counterpart in the reference, whose
   kernels cannot time out. */
gmg_status gmg_coarse_device_error(gmg_coarse* h, int* code);

/* Host copy of the 9-point neighbour table nbr[9][V] (bit-exact index check). */
gmg_status gmg_coarse_neighbors(gmg_coarse* h, int32_t* nbr);

/* Device pointer of the FP64 links in the exchange layout (valid until destroy). */
gmg_status gmg_coarse_links_device(gmg_coarse* h, double** links);

/* ------------------------------------------------------------------------ */
/* Aggregation -- Aggregation (...LutMRHS.h:293-352, AggregationRework.h)    */
/* ------------------------------------------------------------------------ */
typedef struct gmg_agg gmg_agg;

/* Aggregation(CoarseGrid, FineGrid, checkerboard) with site_dof = 12 on the
   fine level or nbasis of the level above for coarse-of-coarse. */
gmg_status gmg_agg_create(const int fine_dims[4], const int coarse_dims[4], int site_dof,
                          int nbasis, gmg_agg** h);
gmg_status gmg_agg_destroy(gmg_agg* h);

/* Upper bound on the basis vectors the coarse-operator construction treats as
   one batch of right-hand sides of the fine operator (0, the default: as many
   as two fine fields of the batch in a third of the free device memory allow,
   at most 40 GB).  A smaller batch trades speed for memory; the links do not
   depend on it.  No counterpart in the reference, which applies the fine
   operator to one basis vector at a time (CoarsenedMatrixUpstream.h:835-844)
   or to batches of Ls vectors, the extent of the fifth (RHS) dimension
   (...LutMRHS.h:1004-1101). */
gmg_status gmg_agg_set_coarsen_batch(gmg_agg* h, int max_batch);

/* subspace[i] = basis[i] (public member `subspace`, ...LutMRHS.h:298). */
gmg_status gmg_agg_set_basis(gmg_agg* h, const double* basis, int on_device, gmg_stream s);
gmg_status gmg_agg_get_basis(gmg_agg* h, double* basis, int on_device, gmg_stream s);

/* Orthogonalise(check, passes) (...LutMRHS.h:318-325) in FP64: per-block
   orthonormalisation, `passes` sweeps (blockLutedOrthonormalise, ...Lut.h:172-240). */
gmg_status gmg_agg_orthonormalise(gmg_agg* h, int passes, gmg_stream s);

/* CheckOrthogonal (...LutMRHS.h:326-340): max over blocks of |B^dag B - 1|_max.
   Synchronises the stream. */
gmg_status gmg_agg_check_orthogonal(gmg_agg* h, double* max_err, gmg_stream s);

/* ProjectToSubspace / PromoteFromSubspace (...LutMRHS.h:341-347), i.e.
   blockLutedInnerProduct / blockLutedAxpy (...Lut.h:70-170) on nrhs RHS.
   fine [Vf][nrhs][dof], coarse [Vc][nrhs][N], both of type vec_prec (F64/F32);
   compute F64 or F32. */
gmg_status gmg_agg_project(gmg_agg* h, gmg_prec compute, gmg_prec vec_prec, int nrhs,
                           const void* fine, void* coarse, gmg_stream s);
gmg_status gmg_agg_promote(gmg_agg* h, gmg_prec compute, gmg_prec vec_prec, int nrhs,
                           const void* coarse, void* fine, gmg_stream s);

/* Chiral doubling of nvec vectors into a 2 nvec basis
   (performChiralDoublingG5C, include/Benchmark_helpers.h:156-181, factor 1/2;
   performChiralDoublingG5R5, :130-154, factor 1): basis[n] = factor (1 + G5)
   v_n and basis[n + nvec] = factor (1 - G5) v_n, G5 = +1 on the upper half of
   the site dof (gamma5 of the chiral basis on spin-colour, G5C on coarse
   vectors).  vecs: device [V][nvec][dof] of prec (F64 / F32, the multi-RHS
   layout of the setup solves); basis: device [2 nvec][V][dof] complex128,
   the layout of gmg_agg_set_basis. */
gmg_status gmg_chiral_double(int64_t V, int dof, int nvec, gmg_prec prec, const void* vecs, double factor,
                             double* basis, gmg_stream s);

/* ------------------------------------------------------------------------ */
/* Fine Wilson-clover operator (Grid WilsonCloverFermionR through            */
/* MdagMLinearOperator::{Op,AdjOp,OpDiag,OpDir}, used at                     */
/* Test_wilsonclover_mg.cc:103-113 and Benchmark_create_coarse_operator.cc)  */
/* ------------------------------------------------------------------------ */
typedef struct gmg_wilson gmg_wilson;

gmg_status gmg_wilson_create(const int dims[4], double mass, double csw, int antiperiodic_t,
                             gmg_wilson** h);
gmg_status gmg_wilson_destroy(gmg_wilson* h);
/* Set the gauge field [V][4][3][3] and build the clover term on the device. */
gmg_status gmg_wilson_set_gauge(gmg_wilson* h, const double* U, int on_device, gmg_stream s);
/* Clover blocks [V][2][6][6] complex128 to host or device memory. */
gmg_status gmg_wilson_get_clover(gmg_wilson* h, double* clover, int on_device, gmg_stream s);
/* op M / Mdag / Mdiag / Mdir(dir, disp); fields [V][nrhs][12] of vec_prec (F64/F32). */
gmg_status gmg_wilson_apply(gmg_wilson* h, gmg_op op, int dir, int disp, gmg_prec vec_prec,
                            int nrhs, const void* in, void* out, gmg_stream s);
/* op M / Mdag in FP64 arithmetic on an FP32 input field, FP64 output: the same
   result as converting in to FP64 and calling gmg_wilson_apply, without the
   converted copy (the FP32 records are promoted exactly on load).  The outer
   FGMRES applies the operator to its FP32 preconditioned directions this way.
   No counterpart (Grid converts between precisions with precisionChange). */
gmg_status gmg_wilson_apply_f32_in(gmg_wilson* h, gmg_op op, int nrhs, const float* in, double* out,
                                   gmg_stream s);
/* out = M in together with the minimal-residual inner products of the MR
   smoother step (the smoother solve of include/MultigridPreconditioner.h:
   264-301): d1[r] = <out_r, in_r>,
   d2[r] = <out_r, out_r> + 0i, device arrays of nrhs complex128.  vec_prec
   F64, F32, or BF16: fields of one 32-bit word per complex number (real part
   in the low 16 bits), FP32 arithmetic, the products from the FP32 result,
   the result rounded to nearest even (the fine smoother of params.smoother_bf16). */
/* Kernel variants of the multi-RHS Wilson-clover apply.  By default the
   variant is autotuned: every applicable one is timed once per (vector
   precision, fused MR products or not, single-hop op or not, nrhs class) on
   the first call that meets the key, and the fastest is kept in the handle.
   gmg_wilson_set_kernel forces one (GMG_WILSON_AUTO restores tuning); a forced
   variant that does not apply to a call falls back to the tuned choice. */
typedef enum {
  GMG_WILSON_AUTO = -1,
  GMG_WILSON_SITE = 0,    /* thread per (site, RHS), operands from global memory */
  GMG_WILSON_TILE = 1,    /* 16-site tiles, links and clover staged in shared memory */
  GMG_WILSON_QUAD = 2,    /* four lanes per (site, RHS), one per spin, quad shuffles */
  GMG_WILSON_STAGED = 3   /* neighbour records bulk-copied into shared memory per tile and RHS chunk */
} gmg_wilson_kernel;
gmg_status gmg_wilson_set_kernel(gmg_wilson* h, gmg_wilson_kernel k);
/* The variant the tuner chose for a key, or GMG_WILSON_AUTO when not tuned yet. */
gmg_status gmg_wilson_tuned_kernel(gmg_wilson* h, gmg_prec vec_prec, int nrhs, int fused_mr, int single_hop,
                                   gmg_wilson_kernel* k);

/* Device error word of this handle's staged (bulk-copy) kernels: 0, or 1 when
   a kernel gave up waiting for its copies; read after a device
   synchronisation and then cleared.  Returns GMG_ERR_TIMEOUT when *code != 0.
   No counterpart in the reference. */
gmg_status gmg_wilson_device_error(gmg_wilson* h, int* code);
gmg_status gmg_wilson_apply_mr(gmg_wilson* h, gmg_prec vec_prec, int nrhs, const void* in, void* out,
                               double* d1, double* d2, gmg_stream s);

/* ------------------------------------------------------------------------ */
/* Gauge-field configuration files (Grid's NerscIO / IldgReader, used at      */
/* src/Test_wilsonclover_mg_lime.cc:57-75, src/Test_wilsonclover_mg.cc:96-99, */
/* NerscIO::writeConfiguration at src/Test_wilson_cg_unprec.cc:72).  Fields   */
/* are host [V][mu][3][3] complex128, sites lexicographic with x fastest: the */
/* layout gmg_wilson_set_gauge takes.                                         */
/* ------------------------------------------------------------------------ */
typedef struct {
  int dims[4];            /* lattice extents from the header */
  int two_row;            /* NERSC 4D_SU3_GAUGE: two rows stored, the third reconstructed */
  int precision;          /* 32 or 64 (bits per real) */
  int big_endian;         /* 1: big-endian payload */
  double plaquette;       /* NERSC header PLAQUETTE (0 if absent) */
  double link_trace;      /* NERSC header LINK_TRACE (0 if absent) */
  uint32_t checksum;      /* NERSC header CHECKSUM */
  uint32_t checksum_data; /* the same sum formed over the payload read */
} gmg_gauge_info;

/* NerscIO::readConfiguration: the header into *info and, when U is not NULL,
   the links into U (V * 36 complex128, from info->dims of a header-only call).
   verify: the checksum, and the plaquette and link trace (formed on the host)
   must match the header (Grid asserts the same three). */
gmg_status gmg_gauge_read_nersc(const char* path, gmg_gauge_info* info, double* U, int verify);
/* NerscIO::writeConfiguration: big-endian IEEE32 or IEEE64 (precision 32 / 64),
   two_row selects 4D_SU3_GAUGE (the third row dropped; exact only for SU(3)
   links) over 4D_SU3_GAUGE_3x3; the header carries the plaquette, link trace
   and checksum. */
gmg_status gmg_gauge_write_nersc(const char* path, const int dims[4], const double* U, int two_row, int precision,
                                 const char* ensemble_id, int sequence_number);
/* IldgReader::readConfiguration: the ildg-format and ildg-binary-data records
   of a LIME file (precision and extents from the format record). */
gmg_status gmg_gauge_read_ildg(const char* path, gmg_gauge_info* info, double* U);
/* Average plaquette Re tr(U_mu U_nu U_mu^dag U_nu^dag) / 3 over sites and the
   six planes, and average link trace Re tr U_mu / 3 (periodic lattice), on the
   GPU; U on the host or the device. */
gmg_status gmg_gauge_plaquette(const int dims[4], const double* U, int on_device, double* plaquette,
                               double* link_trace, gmg_stream s);

/* ------------------------------------------------------------------------ */
/* Galerkin coarse-operator construction                                     */
/* CoarsenOperator(FineGrid, linop, Aggregation) (CoarsenedMatrixUpstream.h: */
/* 755-931, ...DirsaveLut.h:927-1097)                                        */
/* ------------------------------------------------------------------------ */

/* Links of `out` from the fine Wilson-clover operator and the basis of `agg`
   (backward projections + self term by the block even/odd trick + link
   reconstruction), FP64.  The backward hops are evaluated on the face sites
   only, and the self term as one operator pass without the hops between
   blocks of opposite parity.  The first call keeps a workspace in `agg` (two
   fine fields of a batch of basis vectors, at most 40 GB, sized from the free
   memory then) that later calls reuse; it is freed with `agg`.  Asynchronous. */
gmg_status gmg_coarsen_wilson(gmg_coarse* out, gmg_agg* agg, gmg_wilson* fine, gmg_stream s);
/* Coarse-of-coarse: the fine operator is the coarse stencil `fine`. */
gmg_status gmg_coarsen_coarse(gmg_coarse* out, gmg_agg* agg, gmg_coarse* fine, gmg_stream s);

/* ------------------------------------------------------------------------ */
/* Multigrid-preconditioned solve                                            */
/* MultiGridPreconditioner (MultigridPreconditioner.h:44-660, createMGInstance */
/* :665-686) with the outer FGMRES of Test_wilsonclover_mg[_mp].cc            */
/* ------------------------------------------------------------------------ */
typedef struct gmg_mg gmg_mg;

typedef struct {
  int nlevels;           /* 2 or 3 (fine + coarse levels), MultiGridParams::nLevels */
  int block[2][4];       /* aggregation blocks of the transitions 0->1, 1->2 (blockSizes) */
  int nvec[2];           /* test vectors per transition; nbasis = 2 * nvec (chiral doubling) */
  int setup_iters;       /* setup-solver iterations on A psi = v for the test vectors (setupSolverParams) */
  int smoother_iters;    /* MR post-smoothing iterations per level */
  int wrapper_iters;     /* K-cycle FGMRES iterations on intermediate levels (wrapperSolverParams) */
  double wrapper_tol;
  int coarsest_iters;    /* GMRES iterations on the coarsest level (coarsestSolverParams) */
  double coarsest_tol;
  int coarsest_restart;
  int outer_restart;     /* outer FGMRES restart length */
  gmg_prec prec;         /* F64: all FP64; F32: FP32 preconditioner; BF16: FP32 preconditioner with
                            tensor-core coarse stencils.  The outer FGMRES is always FP64. */
  uint64_t seed;         /* test-vector seed */
  int setup_solver;      /* 0: BiCGStab (the reference's default setupSolverType), 1: GMRES(10) */
  double setup_tol;      /* setup-solver tolerance (setupSolverParams.tolerance, 1e-3) */
  int setup_passes;      /* passes over the test vectors (setupInitialIter): each pass solves with the
                            previous pass's vectors (inverse iteration) */
  int setup_null;        /* 1: null-vector setup (setupBasisVectorsType nullVectors: solve A psi = 0 from
                            psi = v); 0: test-vector setup (solve A psi = v from psi = 0) */
  int graph;             /* 1: replay the K-cycle's coarse-level solve (level 1's K-cycle FGMRES and
                            everything below it) as a CUDA graph; the fine level's restriction,
                            prolongation and smoother are plain launches on the Krylov vectors.  The coarse-level
                            solvers keep their Hessenberg / Givens state on the device; each restart
                            cycle and each Arnoldi step is a conditional (IF) node that a device kernel
                            switches on while the level's tolerance and iteration limit are not met,
                            so the replay takes the same early exits as the host-driven cycle.  One
                            graph per active-batch size, captured after one host-driven cycle of that
                            size (default).  0: host-driven cycle (one host synchronisation per
                            Arnoldi step).  The FP64 preconditioner form is always host-driven. */
  int refine_iters[2];   /* refinement setup iterations of the transitions 0->1, 1->2
                            (setupRefinementIter, default {0, 0}); run by gmg_mg_refine */
  int recursive_updates; /* 1: the refinement of a level also replaces the next level's test vectors
                            by its coarse solutions and rebuilds every coarser operator
                            (setupRecursiveUpdates, default 1) */
  int drop_in_cycle;     /* 1 (default): an RHS whose outer FGMRES residual estimate meets the
                            tolerance leaves the batch at that Arnoldi step: the later steps of the
                            cycle apply the preconditioner and the operator to the still-active
                            RHS only.  0: converged RHS leave at the next restart.  No counterpart
                            (the reference solves one RHS at a time). */
  int smoother_bf16;     /* 1: with an FP32 or BF16 preconditioner, the fine level's MR smoother keeps
                            its residual and operator product in BF16 (FP32 arithmetic, FP32
                            solution, the MR inner products from the FP32 operator result), so its
                            sweeps move half the bytes.  0: FP32.  -1 (default): on for the BF16
                            preconditioner form (prec GMG_BF16), off otherwise. */
  int outer_dcgs;        /* 1 (default): the outer FGMRES orthogonalises with delayed
                            reorthogonalisation (the second classical Gram-Schmidt pass of each
                            basis vector merged into the next step): two sweeps over the FP64
                            Krylov basis per step instead of three and a scaling sweep.  0: CGS2. */
  int arnoldi_f32;       /* 1: the outer FGMRES runs each restart cycle's Arnoldi process in FP32
                            (basis, operator products, Gram-Schmidt sweeps; inner products and the
                            Hessenberg least squares in FP64) on the FP64 residual that starts the
                            cycle; the residual b - A x and the solution stay FP64, so every restart
                            is an iterative-refinement step and the tolerance is checked on the FP64
                            true residual.  0: FP64 Arnoldi.  -1 (default): on with an FP32 or BF16
                            preconditioner (prec F32 / BF16), off with prec F64. */
} gmg_mg_params;

/* Defaults of MultiGridParams (MultigridParams.h:95-113) adapted to the MR smoother, with the
   null-vector setup (100 BiCGStab iterations on A psi = 0) instead of one test-vector pass. */
gmg_status gmg_mg_params_default(gmg_mg_params* p);
/* Levels over the fine operator; solves take up to max_rhs right-hand sides at once. */
gmg_status gmg_mg_create(gmg_wilson* fine, const gmg_mg_params* p, int max_rhs, gmg_mg** h);
gmg_status gmg_mg_destroy(gmg_mg* h);
/* initialSetup (MultigridPreconditioner.h:165-211): test vectors, chiral doubling,
   block orthonormalisation and CoarsenOperator on every level.  Synchronises. */
gmg_status gmg_mg_setup(gmg_mg* h, gmg_stream s);
/* refinementSetup (MultigridPreconditioner.h:213-251, BasisVectors.h:74-147 with
   testVectorSetup): for each transition l in order, refine_iters[l] passes of
   {orthonormalise the level's test vectors; replace each by the level-l
   preconditioner (restrict, K-cycle, prolong, smooth) applied to it; with
   recursive_updates, replace the next level's test vector k by the coarse
   solution of that application; orthonormalise; rebuild the aggregation and
   coarse operator of level l (and of every coarser level with
   recursive_updates)}.  As in the reference, a transition with no iterations
   ends the refinement (coarser transitions are not refined).  The test vectors
   of a batch go through the K-cycle together (up to max_rhs at a time).
   Synchronises; operator and aggregation handles keep their addresses. */
gmg_status gmg_mg_refine(gmg_mg* h, gmg_stream s);
/* The preconditioner itself (MultiGridPreconditioner::operator(),
   MultigridPreconditioner.h:253): out = one K-cycle applied to in (restrict,
   coarse K-cycle solve, prolong, MR post-smoothing), computed in the
   preconditioner precision.  in, out: device FP64 [V][nrhs][12], not aliased.
   Synchronises. */
gmg_status gmg_mg_apply(gmg_mg* h, int nrhs, const double* in, double* out, gmg_stream s);
/* Solve D x = b for nrhs right-hand sides with FP64 FGMRES + MG preconditioner to
   per-RHS relative residual |b - D x| / |b| <= tol.  b, x: device FP64
   [V][nrhs][12]; x holds the initial guess.  Converged RHS drop out at the
   Arnoldi step their residual estimate meets tol (params.drop_in_cycle), and
   at every outer restart by their true residual.  Synchronises;
   GMG_ERR_NOT_CONVERGED if maxiter is reached. */
gmg_status gmg_mg_solve(gmg_mg* h, int nrhs, const double* b, double* x, double tol, int maxiter, int* iters,
                        double* max_relres, gmg_stream s);
/* Per-RHS outcome of the last gmg_mg_solve on this handle (nrhs must be that
   solve's): iters[r], the outer iteration at which RHS r's residual estimate
   met tol (the last count reached if it never did), and relres[r], its true
   relative residual at the end.  No
   counterpart: the reference solves one RHS per solver call and times it
   (Test_wilsonclover_mg.cc:140-151). */
gmg_status gmg_mg_solve_stats(gmg_mg* h, int nrhs, int* iters, double* relres);
/* The active-batch size of every outer Arnoldi step of the last gmg_mg_solve
   (the RHS the preconditioner and the operator were applied to): *n steps,
   the first min(cap, *n) written to sizes.  No counterpart. */
gmg_status gmg_mg_solve_batches(gmg_mg* h, int cap, int* sizes, int* n);
/* Captured K-cycle graphs of this handle (params.graph): how many (one per
   active-batch size met so far) and whether a capture failed, in which case
   the solver kept the host-driven cycle.  No counterpart in the reference. */
gmg_status gmg_mg_graphs(gmg_mg* h, int* graphs, int* fell_back);
/* The coarse operator of level > 0 and the aggregation from level to level+1
   (runChecks, MultigridPreconditioner.h:311-446); either may be null. */
gmg_status gmg_mg_level(gmg_mg* h, int level, gmg_coarse** op, gmg_agg** agg);

/* ------------------------------------------------------------------------ */
/* Rework layout maps (Layout_converters.h:33-139): flat basis index          */
/* n = s*Nc_c + c <-> (s, c).  Device links [V][N][N], inverse=1 for spin->flat */
/* ------------------------------------------------------------------------ */
gmg_status gmg_layout_links(int64_t V, int nbasis, int ncs, const double* in, double* out,
                            int inverse, gmg_stream s);
/* Rework layout map of coarse vectors (Layout_converters.h:92-139): flat
   basis index n = s*Nc_c + c <-> (s, c), rows = sites x nrhs.  In the
   lexicographic [row][N] buffers of this library both forms have the same
   memory order, so the map is a copy; it is kept as an entry so that an
   adapter converting Grid fields calls it where the reference calls
   convertLayout. */
gmg_status gmg_layout_vectors(int64_t rows, int nbasis, int ncs, const double* in, double* out,
                              int inverse, gmg_stream s);

/* ------------------------------------------------------------------------ */
/* Two-spin (Rework) forms of the subspace and of the links                  */
/* (CoarseningPolicyRework.h:56-109, AggregationRework.h:75-146,             */
/* CoarsenedMatrixRework.h:60-101).  The Rework classes keep                 */
/* Nc_c = nbasis / ncoarse_spins basis vectors; coarse component (s, c) is   */
/* the projection on the part of vector c on the s-th of ncoarse_spins equal */
/* slices of the fine site dof (the two chiralities of a Wilson spinor, the  */
/* G5C halves of a coarse vector).  This library stores that as the doubled  */
/* basis with flat index n = s * Nc_c + c, so coarse vectors are the same    */
/* memory in both forms; subspace and links are converted by these entries.  */
/* ------------------------------------------------------------------------ */
/* subspace_[c] = vecs[c] (Rework::Aggregation::Create's copy, :127-146):
   vecs [Nc_c][Vf][dof] complex128; basis vector s * Nc_c + c becomes the
   part of vecs[c] on dof slice s (zero elsewhere). */
gmg_status gmg_agg_set_subspace_spins(gmg_agg* h, int ncoarse_spins, const double* vecs, int on_device,
                                      gmg_stream s);
/* Rework::Aggregation::Subspace() (:75-76): vecs[c] = sum_s basis[s * Nc_c + c]. */
gmg_status gmg_agg_get_subspace_spins(gmg_agg* h, int ncoarse_spins, double* vecs, int on_device, gmg_stream s);
/* Rework::CoarsenedMatrix::Y_[point] (:70): links [V][Ns_c][Ns_c][Nc_c][Nc_c]
   complex128, Y(s1, s2)(c1, c2) = A_point[s1 Nc_c + c1][s2 Nc_c + c2]
   (convertLayout, Layout_converters.h:33-90). */
gmg_status gmg_coarse_get_links_spins(gmg_coarse* h, int ncoarse_spins, int point, double* links, int on_device,
                                      gmg_stream s);
/* All nine Y_[p] in that form, [9][V][Ns_c][Ns_c][Nc_c][Nc_c] (as gmg_coarse_set_links). */
gmg_status gmg_coarse_set_links_spins(gmg_coarse* h, int ncoarse_spins, const double* links, int on_device,
                                      gmg_stream s);

/* ------------------------------------------------------------------------ */
/* Live kernel timing (replaces the reference's Profiler stopwatches,        */
/* include/Profiler.h:153-296, with CUDA events on the launching stream)     */
/* ------------------------------------------------------------------------ */
/* Enable / disable event recording around the hot kernels. */
gmg_status gmg_profile_enable(int on);
/* Summed device time and launch count of one kernel since the last read, then
   reset.  Names: "coarse_mrhs_tc", "coarse_simt", "wilson", "project",
   "promote", "ortho".  Synchronises the recorded events. */
gmg_status gmg_profile_read(const char* kernel, double* total_ms, int64_t* launches);

#ifdef __cplusplus
}
#endif
#endif /* GMG_H */
