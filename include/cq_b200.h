/*
 * cq_b200.h -- C ABI of the B200-native CONQUEST block-sparse multiply and
 * LNV / McWeeny density-matrix solver (libcqb200.so).
 *
 * Conventions shared with the reference (OrderN/CONQUEST-release):
 *   - A block-sparse matrix of range r is one flat FP64 array holding, for each
 *     primary atom i (partition order) and each neighbour j within r (covering
 *     set order, periodic images distinct), an nd_i x nd_j block stored column
 *     major (i orbital fastest).  This is the storage of `mat_p(A)%matrix`
 *     (src/mult_module.f90) built by get_naba / make_halo
 *     (src/matrix_elements_module.f90:257-716).
 *   - mult_type 1 computes C = A.B (C overwritten); mult_type 2 computes
 *     a = c.b^T restricted to the range of a (a overwritten), with the argument
 *     roles of mat_mult (src/multiply_module.f90:115).
 *   - Every entry point returns 0 on success or a CQ_ERR_* code; the message of
 *     the last failure is returned by cq_last_error().  The Fortran shim maps a
 *     nonzero status to cq_abort (src/GenComms/generic_comms.f90:95).
 *
 * Pointers named *_dev are device (HBM) pointers; every other pointer is host
 * memory.  Calls on one system are stream ordered and not re-entrant.
 */
#ifndef CQ_B200_H
#define CQ_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CQ_OK 0
#define CQ_ERR_ARG 1          /* invalid argument or unknown range / product */
#define CQ_ERR_OOM 2          /* device allocation failed */
#define CQ_ERR_CUDA 3         /* CUDA runtime error */
#define CQ_ERR_BOUNDS 4       /* an index check failed (the kernel skipped the access) */
#define CQ_ERR_TIMEOUT 5      /* a bounded wait ran out */
#define CQ_ERR_STATE 6        /* call not valid in the current state */
#define CQ_ERR_NOT_CONVERGED 7
#define CQ_ERR_CALLBACK 8     /* a caller-supplied callback returned nonzero */

typedef struct cq_system cq_system;

/* Last error message of the calling thread (static storage, never NULL). */
const char* cq_last_error(void);

/* Library version string. */
const char* cq_version(void);

/*
 * Geometry and index construction for one periodic system on one GPU.
 * Replaces the one-process path of sfc_partitions_to_processors
 * (src/sfc_partitions_module.f90:124), make_prim (src/primary_module.f90:97),
 * make_cs (src/cover_module.f90:133) and matrix_ini for every listed range
 * (src/matrix_elements_module.f90:67-142, called from immi,
 * src/mult_module.f90:271).  The covering set is built for the largest range.
 *   coords[3*n]  Cartesian positions (bohr), wrapped into the cell as
 *                read_atomic_positions does (src/io_module.f90:418)
 *   cell[3]      orthorhombic cell lengths
 *   nsf[n]       block size (support functions) of each atom
 *   rcuts[n_ranges] matrix ranges; range r is addressed by its position
 *   max_atoms_part General.MaxAtomsPartition (reference default 34)
 *   gap_threshold, avg_atomic_diameter  General.GapThreshold / AverageAtomicDiameter
 * The neighbour lists, halos, retro lists and transposes are built on the GPU.
 */
int cq_system_create(int n_atoms, const double* coords, const double* cell, const int* nsf, int n_ranges,
                     const double* rcuts, int max_atoms_part, double gap_threshold, double avg_atomic_diameter,
                     cq_system** out);
/* Fails with CQ_ERR_STATE, destroying nothing, while LNV solvers built on the system are alive:
 * destroy those (cq_lnv_destroy) first. */
int cq_system_destroy(cq_system* sys);

/* Number of stored elements (mat_p(A)%length) and blocks of range r. */
int cq_range_length(cq_system* sys, int r, int64_t* length, int64_t* n_blocks);

/*
 * Export one index array of range r (r < 0: a geometry array) as int64, in the
 * reference's 1-based conventions, for bit-exact parity checks.  Names:
 *   geometry: "n_parts", "cover_dims", "ngnode", "nm_group", "ig_prim",
 *             "lab_cell", "lab_cover", "n_ing_cover", "icover_ibeg", "ig_cover", "iprim_group"
 *   range:    "n_nab", "i_acc", "i_nd_acc", "ndimi", "onsite", "i_part", "i_seq",
 *             "ndimj", "npxyz", "bind", "halo_sizes", "nh_part", "j_beg",
 *             "lab_hcell", "lab_hcover", "j_seq", "halo_ndimj", "i_halo", "i_h2d",
 *             "t_i_prim", "t_i_beg", "t_i_nd_beg", "t_n_hnab", "itran_addr"
 * With out == NULL only *n is set.
 */
int cq_export_index(cq_system* sys, int r, const char* name, int64_t* out, int64_t cap, int64_t* n);

/* Radii of the stored blocks of range r (matrix%radius), nnz entries. */
int cq_export_radius(cq_system* sys, int r, double* out, int64_t cap, int64_t* n);

/*
 * mat_mult on device-resident operands (src/multiply_module.f90:115-359 with
 * the m_kern_max / m_kern_min summation order of
 * src/multiply_kernel_default.f90:132-224, 325-412).
 *   mult_type 1: c_dev (range rc) = a_dev (range ra) . b_dev (range rb)
 *   mult_type 2: a_dev (range ra) = c_dev (range rc) . b_dev^T (range rb)
 * `precision` selects the arithmetic:
 *   CQ_PREC_FP64 (1): FP64 with the reference's separate multiply and add per
 *     term, bit-identical to the default kernel built without FMA contraction;
 *   CQ_PREC_FP64_FMA (0): FP64 with fused multiply-add;
 *   CQ_PREC_BF16X3 (2): blocks padded to 16 x 16 and split v = hi + lo in bf16,
 *     hi.hi + hi.lo + lo.hi on the tensor cores with FP32 accumulation, stored
 *     back as FP64 (about 16 significant bits per product term);
 *   CQ_PREC_BF16X6 (3): blocks padded to 16 x 16 and split v = hi + mid + lo in
 *     bf16, six products per block pair (hi.hi, hi.mid, mid.hi, hi.lo, lo.hi,
 *     mid.mid) on the tensor cores (mma.sync), each pair's product rounded once
 *     to FP32 and the pairs summed in FP64 (about 22 significant bits per term);
 *   CQ_PREC_FP64_TC (4): FP64 on the tensor cores (mma.sync.m8n8k4.f64, blocks
 *     padded to 16 x 16): each MMA chains its products as fused multiply-adds in
 *     the terms' order, so the result has the bits of CQ_PREC_FP64_FMA (measured
 *     on B200), which runs this way for blocks larger than 8 x 8.
 * The pair lists of the product are built on the first call and cached.  Work
 * is enqueued on the system's stream; the call returns without synchronising.
 */
#define CQ_PREC_FP64_FMA 0
#define CQ_PREC_FP64 1
#define CQ_PREC_BF16X3 2
#define CQ_PREC_BF16X6 3
#define CQ_PREC_FP64_TC 4
int cq_mat_mult(cq_system* sys, int mult_type, int ra, int rb, int rc, double* a_dev, const double* b_dev,
                double* c_dev, int precision);

/*
 * Batched products (no counterpart in the reference, which runs one mat_mult at a time): n
 * independent FP64 products (precision[k] CQ_PREC_FP64 or CQ_PREC_FP64_FMA), each on its own system
 * or on one system with different operands, run as ONE persistent kernel over the concatenation of
 * their output-block lists.  Product k has the arguments of cq_mat_mult on systems[k].  Every output
 * element sees the same operations as in cq_mat_mult, so the results are bit-identical to n separate
 * calls.  The launch is enqueued on systems[0]'s stream after the work already enqueued on every
 * system's stream, and later work on every system's stream waits for it.  The call waits for the
 * copy of the launch's small descriptor table (not for the products).
 */
int cq_mat_mult_batch(int n, cq_system* const* systems, const int* mult_type, const int* ra, const int* rb,
                      const int* rc, double* const* a_dev, const double* const* b_dev, double* const* c_dev,
                      const int* precision);

/* Same as cq_mat_mult with host arrays: copies in, multiplies, copies the result out, synchronises. */
int cq_mat_mult_host(cq_system* sys, int mult_type, int ra, int rb, int rc, double* a, const double* b, double* c,
                     int precision);

/*
 * Matrices by id: the HBM side of mat_p(id)%matrix (src/matrix_data_module.f90).  The system owns
 * one device copy per bound id, in the block layout of the id's range; the caller's host array
 * (mat_p(id)%matrix) is copied on demand.  The operations mirror mult_module's by-index calls
 * (matrix_product, matrix_sum, matrix_transpose, matrix_product_trace; src/mult_module.f90:
 * 2556-2916) on those device copies, enqueued on the system's stream.
 *   cq_matrix_bind      allocate the zeroed device copy of id in range r; host (range length
 *                       doubles, may be NULL) is remembered, not copied; an id binds once
 *   cq_matrix_unbind    release it (on the system's current stream, after the work enqueued there)
 *   cq_matrix_device    its device pointer and length (for cq_mat_mult and the other entries)
 *   cq_matrix_upload    host -> device, stream-ordered: the call returns once the copy is queued,
 *                       so the host array must stay unchanged (and allocated) until the next call
 *                       on the system that synchronises (cq_matrix_download, cq_synchronize);
 *                       cq_matrix_download device -> host (synchronises)
 *   cq_matrix_product_id  mult_type 1: idc = ida . idb; 2: ida = idc . idb^T (ranges from the
 *                       bound ids; the output must not be an input)
 *   cq_matrix_sum_id    ida = alpha ida + beta idb (any two ranges, as matrix_sum)
 *   cq_matrix_transpose_id / cq_matrix_product_trace_id  as cq_matrix_transpose / _product_trace
 */
int cq_matrix_bind(cq_system* sys, int id, int r, double* host);
int cq_matrix_unbind(cq_system* sys, int id);
int cq_matrix_device(cq_system* sys, int id, double** dev, int64_t* length);
int cq_matrix_upload(cq_system* sys, int id);
int cq_matrix_download(cq_system* sys, int id);
int cq_matrix_product_id(cq_system* sys, int mult_type, int ida, int idb, int idc, int precision);
int cq_matrix_sum_id(cq_system* sys, int ida, double alpha, int idb, double beta);
int cq_matrix_transpose_id(cq_system* sys, int ida, int idat);
int cq_matrix_product_trace_id(cq_system* sys, int ida, int idb, double* result);

/*
 * Matrix files in the reference's binary format (dump_matrix2 / grab_matrix2,
 * src/store_matrix_module.f90:340-430, 1199-1421: Fortran unformatted sequential records; one
 * file per process, here one): the device array a_dev of range r is written with its block
 * layout (global ids, neighbours' block sizes, fractional image vectors) or read back.  Reading
 * matches every block of the file to a block of the range by (global i, global j, image vector);
 * blocks of the range absent from the file become zero; *matched receives the number of matched
 * file blocks.  Restart and persistence of L (`Lmatrix2` files).
 */
int cq_dump_matrix(cq_system* sys, int r, const double* a_dev, const char* path, int inode);
int cq_grab_matrix(cq_system* sys, int r, double* a_dev, const char* path, int64_t* matched);

/* Algorithmic work of one product: (k,i,j) triples with a stored result and 2*sum nd^3 flops. */
int cq_product_work(cq_system* sys, int mult_type, int ra, int rb, int rc, int64_t* triples, int64_t* flops);

/* Autotuner record of one product: the FP64 kernel variant it chose (-1 before the product's
 * first autotuned call) and the timed milliseconds of each candidate variant (ms[7], 0 = not
 * timed); for its split-precision form the output blocks per warp it chose (1, 2, 4 or 8; -1 =
 * not tuned yet) and the timed milliseconds of those four group sizes (group_ms[4]). */
int cq_product_tuning(cq_system* sys, int mult_type, int ra, int rb, int rc, int* variant, float* ms, int* group,
                      float* group_ms);

/* Tensor-core form of one product (no counterpart in the reference, whose kernels are scalar): the
 * dense 128 x 128 tiles its split-precision products run on (building their plan on first use),
 * the tensor work those tiles issue (3 MMAs x 2 x 128 x 128 x the K extent padded to the pipeline's
 * chunk, per tile), and whether every block size fits the tiles (4..128; usable = 0: the
 * split-precision products of this system run one padded block per warp instead). */
int cq_product_tensor_work(cq_system* sys, int mult_type, int ra, int rb, int rc, int64_t* tiles,
                           int64_t* issued_flops, int* usable);

/*
 * Drop-in kernel pair (plugin surface of multiply_kernel_<MULT_KERN>.f90):
 * the argument lists of m_kern_max / m_kern_min
 * (src/multiply_kernel_default.f90:132-160, 325-358) with the derived types
 * flattened into their component arrays (Fortran 1-based values, host memory):
 *   ahalo: nh_part, j_beg, j_seq, ndimi, ndimj
 *   chalo: i_halo, i_hbeg, i_h2d (n_prim*ni_in_halo), ni_in_halo
 *   at   : i_prim, i_beg, i_nd_beg, n_hnab
 * a(lena) is the local transpose (type 1) or the accumulator (type 2),
 * b(lenb) the partition's B data, c(lenc) the accumulator (type 1) or input
 * (type 2); the accumulator is updated in place on return, exactly as one call
 * of the default kernel for partition kpart.
 */
int cq_m_kern_max(int k_off, int kpart, const int* ib_nd_acc, const int* ibaddr, const int* nbnab, const int* ibpart,
                  const int* ibseq, const int* bndim2, const double* a, const double* b, double* c,
                  const int* ahalo_nh_part, const int* ahalo_j_beg, const int* ahalo_j_seq, const int* ahalo_ndimi,
                  const int* ahalo_ndimj, const int* chalo_i_halo, const int* chalo_i_hbeg, const int* chalo_i_h2d,
                  int chalo_ni_in_halo, const int* at_i_prim, const int* at_i_beg, const int* at_i_nd_beg,
                  const int* at_n_hnab, int mx_absb, int mx_part, int mx_iprim, int lena, int lenb, int lenc);
int cq_m_kern_min(int k_off, int kpart, const int* ib_nd_acc, const int* ibaddr, const int* nbnab, const int* ibpart,
                  const int* ibseq, const int* bndim2, double* a, const double* b, const double* c,
                  const int* ahalo_nh_part, const int* ahalo_j_beg, const int* ahalo_j_seq, const int* ahalo_ndimi,
                  const int* ahalo_ndimj, const int* chalo_i_halo, const int* chalo_i_hbeg, const int* chalo_i_h2d,
                  int chalo_ni_in_halo, const int* at_i_prim, const int* at_i_beg, const int* at_i_nd_beg,
                  const int* at_n_hnab, int mx_absb, int mx_part, int mx_iprim, int lena, int lenb, int lenc);

/* Deferred drop-in calls (no counterpart in the reference, whose kernels return with their result in
 * c): with np_in_halo > 0 (the A halo's partition count, ahalo%np_in_halo, which the Fortran shim
 * passes before every m_kern call) the cq_m_kern_max / cq_m_kern_min calls of one mat_mult partition
 * loop keep a and c on the device from the first partition (kpart == 1) on, copy only their
 * partition's b and block lists, enqueue their arithmetic and return; the call with
 * kpart == np_in_halo copies the result (c for m_kern_max, a for m_kern_min) back to the array the
 * first partition's call passed and synchronises.  a and c must not change between the calls of
 * one loop (mat_mult does not change them).  cq_m_kern_flush completes an open loop at once;
 * cq_m_kern_defer(0) flushes and returns to complete-per-call.  Per calling thread.  Results are
 * bit-identical to complete-per-call. */
int cq_m_kern_defer(int np_in_halo);
int cq_m_kern_flush(void);

/* matrix_sum (src/mult_module.f90:2677-2715): a = alpha*a + beta*b; ranges may differ (matrix_add rules). */
int cq_matrix_sum(cq_system* sys, int ra, double* a_dev, double alpha, int rb, const double* b_dev, double beta);
/* matrix_transpose within one range (src/mult_module.f90:2609-2673). */
int cq_matrix_transpose(cq_system* sys, int r, const double* a_dev, double* at_dev);
/* matrix_trace (src/mult_module.f90:2773-2811) and matrix_product_trace (2885-2916). */
int cq_matrix_trace(cq_system* sys, int r, const double* a_dev, double* result);
int cq_matrix_product_trace(cq_system* sys, int r, const double* a_dev, const double* b_dev, double* result);

/* Synchronise the system's stream. */
int cq_synchronize(cq_system* sys);

/* Enqueue all further work of the system on `stream` (a cudaStream_t); NULL restores its own stream.
 * The call synchronises the previous stream first.  A stream given here must stay valid until the
 * system (and every solver on it) is destroyed: buffers allocated while it was current are released
 * on it. */
int cq_system_set_stream(cq_system* sys, void* stream);

/* CUDA-event timing of every block-product launch (timer_module's tmr_std_matmult, per launch). */
int cq_profile_enable(cq_system* sys, int on);
/* Synchronise, return and reset: timed product launches, their total milliseconds, algorithmic
 * bytes (8 * (len A + len B + len C) per launch) and flops (2 sum nd^3 over the triples). */
int cq_profile_read(cq_system* sys, int64_t* launches, double* ms, double* bytes, double* flops);
/* Kernels launched by this system so far (all kinds). */
int cq_launch_count(cq_system* sys, int64_t* count);

/* Synthetic input generator (no counterpart in the reference, whose S and H come from grid
 * integration): writes S (which = 0: onsite identity, offsite 0.3 exp(-r/2)) or H (which = 1:
 * onsite diagonal -0.5 u(seed, atom, orbital), offsite -0.2 exp(-r/2)) of range r into the device
 * array `out` (range length), stream-ordered.  Same values as cq_b200.inputs.overlap_S /
 * hamiltonian_H up to the last bit of exp(). */
int cq_generate_SH(cq_system* sys, int r, int which, uint64_t seed, double* out);

/* Tuning options.  CQ_OPT_MULT_VARIANT: FP64 4x4 product kernel, -1 = chosen per product by the
 * autotuner (default: the first call of each product times the candidate kernels with CUDA
 * events and keeps the fastest), 0 = one lane per output element, 1 = one thread per output
 * block, 2 = one thread per output block with the first operand's row staged in shared memory,
 * 3 = one thread per output block with the warp staging the operand blocks through shared
 * memory, 5 = four lanes per output block (one column each), the first operand's block staged
 * in shared memory, 6 = one thread per output block with its operand blocks staged by bulk copies
 * (cp.async.bulk, completion on an mbarrier, bounded waits); for other block sizes (DZP 13 x 13,
 * mixed sizes) 0 = one warp per output block, one lane per element, 4 = one warp per output block,
 * a 4 x 2 register tile per lane (the autotuner candidates are 3/5/1/0 for uniform 4 x 4 blocks
 * and 4/0 otherwise; variant 6 is selectable only).  All give
 * identical results.
 * CQ_OPT_BLOCKING_SYNC: 1 = the host thread sleeps on a blocking-sync event whenever the
 * solver waits for a scalar from the device (many concurrent solvers per host core), 0 = it
 * spins in cudaStreamSynchronize (default, lowest latency for one solver). */
#define CQ_OPT_MULT_VARIANT 1
#define CQ_OPT_BLOCKING_SYNC 2
/* CQ_OPT_MIXED_KERNEL: kernel of the CQ_PREC_BF16X3 products (CQ_PREC_BF16X6 products always run on
 * mma.sync: the tcgen05 tiles accumulate a whole contraction in FP32).  -1 (default) = chosen per product
 * by a fixed rule (the tiles where at least 11 % of their issued tensor work is useful), so a product
 * always gives the same bits; 0 = dense 128 x 128 tiles on the tcgen05 tensor cores with TMEM
 * accumulators, operands staged by bulk copies (every block size 4..16; other systems use 1);
 * 1 = one padded 16 x 16 block per warp-level mma.sync. */
#define CQ_OPT_MIXED_KERNEL 3
/* CQ_OPT_TEST_STALL (test hook): 1 = in the next tensor-core product the bulk-copy thread stops after
 * taking its first tile, so the kernel's bounded waits run out (about a second) and the call that
 * synchronises (cq_mat_mult_host, cq_synchronize, the chain's waits) returns CQ_ERR_TIMEOUT; the
 * context stays usable and the product's output is not valid.  One product, then back to 0. */
#define CQ_OPT_TEST_STALL 4
/* CQ_OPT_SPLIT_GROUP: output blocks per warp of the mma.sync split-precision kernels.  -1 (default)
 * = chosen per product by the autotuner; 1, 2, 4 (and 8, two-part split only) = that group size.
 * Every group size gives the same bits (each output block sums its own terms in its own order). */
#define CQ_OPT_SPLIT_GROUP 5
int cq_system_set_option(cq_system* sys, int option, int value);

/* ------------------------------------------------------------------------ */
/* LNV / McWeeny density-matrix minimisation (one spin channel, nspin = 1)   */
/* ------------------------------------------------------------------------ */
typedef struct cq_lnv cq_lnv;

/* Control parameters; defaults are the reference's fdf defaults
 * (src/initial_read_module.f90:1208, 1598-1608, 1901-1904). */
typedef struct {
  int n_L_iterations;      /* DM.LVariations (50) */
  double tolerance;        /* minE.LTolerance (1e-7) */
  int maxpulay;            /* DM.MaxPulay (5) */
  double minpulaystep;     /* DM.MinPulayStepSize (1e-3) */
  double maxpulaystep;     /* DM.MaxPulayStepSize (0.1) */
  double lintol;           /* DM.LinTol (0.1) */
  int global_tolerance;    /* minE.GlobalTolerance (0 for static runs) */
  int vary_mu;             /* !DM.ConstantMu (1) */
  int invs_max_steps;      /* DM.InvSMaxSteps (100) */
  double invs_delta_tol;   /* DM.InvSDeltaOmegaTolerance (1e-4) */
  double invs_tol;         /* DM.InvSTolerance (1e-2) */
  int exact;               /* 1: FP64 products with the default kernel's rounding; 0: fused multiply-add */
  int max_outer;           /* bound on FindMinDM outer passes (40); the reference loops until done, which a
                              residual stalled above `tolerance` never reaches: the solve then stops with
                              converged = 0 */
  int mixed;               /* 1: cq_lnv_solve runs FindMinDM (McWeeny start included) with split-precision
                              products (split_parts) to `mixed_tolerance` (at most mixed_max_outer passes),
                              then continues from that L with FP64 products to `tolerance`;
                              Hotelling, traces, line search and Pulay stay FP64 */
  double mixed_tolerance;  /* residual at which the split-precision phase hands over to FP64; <= 0
                              (default): max(tolerance, 1e-8) for split_parts 3, 1e-6 for split_parts 2 */
  int fp64_mcw_sweeps;     /* FP64 McWeeny purification sweeps of L between the two phases (0) */
  int graphs;              /* 1: each LNV_matrix_multiply call is captured once in a CUDA graph and replayed
                              (same results; default 1) */
  int mixed_mcw;           /* mixed form: 1 = the McWeeny start also runs split-precision products
                              (default 0: FP64, the same start as the FP64 solve) */
  int fp64_continue;       /* mixed form: 1 = FindMinDM continues in FP64 to `tolerance` (default);
                              0 = after the split-precision phase only the FP64 purification sweeps
                              (fp64_mcw_sweeps) and an FP64 evaluation of K, energy and electrons */
  int split_parts;         /* mixed form: bf16 parts per value of the split-precision products,
                              2 = CQ_PREC_BF16X3, 3 = CQ_PREC_BF16X6 (default); 0 = no split-precision
                              phase (with fp64_tensor: every product on the FP64 tensor cores) */
  int mixed_max_outer;     /* mixed form: FindMinDM passes of the split-precision phase (always leaving
                              at least one of max_outer to FP64); 0 (default) = 2 for split_parts 2,
                              4 for split_parts 3 */
  int fp64_tensor;         /* mixed form: 1 (default) = its FP64 products of blocks larger than 8 x 8
                              (McWeeny start, Hotelling, the FP64 continuation) run as CQ_PREC_FP64_TC,
                              the bits of fused multiply-add FP64; 0 = as `exact` */
} cq_lnv_params;

typedef struct {
  double energy;           /* band energy 2 Tr(K H), K = 3LSL - 2LSLSL */
  double electrons;        /* 2 (3 Tr(L SLS) - 2 Tr(L SLSLS)) */
  double residual;         /* last DM residual g (per atom unless global_tolerance) */
  double invs_omega;       /* Hotelling residual of T = S^-1 */
  int mcw_sweeps, early_iters, late_iters, ne_corrections, inflexions, converged;
  int outer_iters;         /* FindMinDM passes (early + late) run */
  int64_t graph_launches;  /* LNV_matrix_multiply calls replayed from a CUDA graph */
  int64_t n_products;      /* block-sparse products executed */
  int64_t flops;           /* algorithmic flops of those products (2 sum nd_i nd_j nd_k) */
  int64_t n_products_mixed;/* of which with split-precision tensor-core arithmetic */
  int64_t flops_mixed;
  int split_restarts;      /* mixed form: 1 if the split-precision phase stalled more than 100 times
                              above its hand-over residual and the FP64 phase started again from the
                              McWeeny start */
} cq_lnv_result;

int cq_lnv_params_default(cq_lnv_params* p);

/*
 * Density-matrix solver on a system.  ranges[11] gives the system range index
 * of S, H, L, T, LS, LH, LSL, SLS, TS, TH, TL in that order (rcut(LS) = L + S,
 * rcut(LSL) = 2L + S ... as src/dimens_module.f90:338-355; SL, HL, LTr, TTr
 * share the index of LS, LH, L, T).  ne_spin = ne_spin_in_cell(1).
 */
int cq_lnv_create(cq_system* sys, const int* ranges, double ne_spin, const cq_lnv_params* p, cq_lnv** out);
int cq_lnv_destroy(cq_lnv* s);
/* Load S and H (range layouts of S and H) from host or device memory. */
int cq_lnv_set_SH(cq_lnv* s, const double* S, const double* H, int on_device);
/* T = S^-1 by Hotelling iterations (Iter_Hott_InvS, src/S_matrix_module.f90:746-963); omega returned. */
int cq_lnv_invert_S(cq_lnv* s, double* omega);
/* FindMinDM (src/DMMinModule.f90:172-312); resetL != 0 starts from the McWeeny initial L. */
int cq_lnv_find_min_dm(cq_lnv* s, int resetL, cq_lnv_result* res);
/* Copy one matrix out: name in "L", "K", "T", "S", "H", "phi"; to host (on_device = 0) or device memory. */
int cq_lnv_get(cq_lnv* s, const char* name, double* out, int64_t cap, int on_device);
/* Copy a matrix in (for example a previous L): name in "L", "T". */
int cq_lnv_put(cq_lnv* s, const char* name, const double* in, int on_device);
/*
 * DoPulay2D_nospin (src/Pulay.f90:188-262): Pulay mixing coefficients from the
 * n x n residual overlap Aij (column major, leading dimension max_n), inverted by
 * Bunch-Kaufman pivoting as LAPACK dsytf2/dsytri; if a pivot is singular alphas is
 * the unit vector e_ipulay.  Host-only, needs no GPU.
 */
int cq_pulay_alphas(int ipulay, const double* Aij, int n, int max_n, double* alphas);
/* SolveCubic (src/DMMinModule.f90:2072-2143): a real root of x^3 + a x^2 + b x + c = 0 by
 * Cardano's formula, the one of least magnitude when there are three; with one real root farther
 * than 10 |guess| from zero, guess.  The root the electron-number correction steps to.  Host-only,
 * needs no GPU. */
int cq_solve_cubic(double a, double b, double c, double guess, double* x);

/* One complete solve on the device-resident S and H: T = S^-1, then FindMinDM from the McWeeny start. */
int cq_lnv_solve(cq_lnv* s, cq_lnv_result* res);
/*
 * One complete solve from host arrays: load S and H, T = S^-1, FindMinDM from
 * the McWeeny start, copy L and K back (either may be NULL).  This is the
 * end-to-end call of a user holding S and H in host memory.
 */
int cq_lnv_solve_host(cq_lnv* s, const double* S, const double* H, double* L_out, double* K_out, cq_lnv_result* res);

/*
 * Exact dot products that allocate nothing (no counterpart in the reference).  For callers that
 * cannot allocate device memory when they need a trace: a Fortran/MPI host that has handed the
 * whole device to its own memory pool, or a latency-critical loop that must not take the
 * device-wide synchronisation cudaMalloc/cudaFree can imply.  out[k] = sum_i x_dev[k][i] *
 * y_dev[k][i] over n[k] elements (a plain sum where y_dev is NULL or y_dev[k] is NULL), with the
 * same exact, order-independent rounding as cq_matrix_product_trace, so the values are
 * bit-identical to it.  x_dev / y_dev are host arrays of device pointers; work is enqueued on
 * `stream` (a cudaStream_t, NULL = the default stream) and the call synchronises it.
 *   - At most CQ_NOALLOC_MAX_SUMS sums per call; more is rejected with CQ_ERR_ARG.
 *   - The scratch is one static device array of 28.7 KiB that every GPU loading the library
 *     holds until exit.  Every call looks up that array's device address on the current device
 *     (the first lookup on a device may load the library's device code there: make the first
 *     call before any stream capture on that device).
 *   - Every call shares the array: calls that overlap on the GPU (two streams, two threads) race
 *     and give wrong sums.  Serialise them.
 */
#define CQ_NOALLOC_MAX_SUMS 8
int cq_exact_dots_noalloc(int count, const double* const* x_dev, const double* const* y_dev, const int64_t* n,
                          void* stream, double* out);

/* Force matrices of the current L (the doM1 + doM2 and doM4 branches of LNV_matrix_multiply,
 * src/mult_module.f90:1564-1592, 1680-1726), FP64 with the reference's rounding:
 *   M12 = 3 LHL - 2 LHLSL - 2 LSLHL  (S range; LHL = LH.L in the SLS range, LHLSL = LHL.SL pruned
 *                                      to the S range, LSLHL its transpose)
 *   M4  = 12 LSL - 12 LSLSL          (H range)
 * Either output may be NULL.  on_device: the outputs are device arrays. */
int cq_lnv_force_matrices(cq_lnv* s, double* M12, double* M4, int on_device);

/*
 * Mixed-L self-consistency (minE.MixedLSelfConsistent, src/DMMinModule.f90:894-907, 1138-1149):
 * with a callback set, lateDM rebuilds H from the density of the current L at its start and after
 * every Pulay step, as the reference does with get_electronic_density + get_H_matrix; the
 * residual-rise exit of lateDM is then off (DMMinModule.f90:1261).  Each rebuild first evaluates
 * K = 3LSL - 2LSLSL and Tr(KH) of the current L (LNV_matrix_multiply with doK, doE), then calls
 *   fn(user, K_dev, H_dev, length, stream)
 * on the solving thread: K_dev and H_dev are the solver's device arrays of K and H (both the H
 * range, `length` doubles), `stream` is the solver's cudaStream_t.  The callback writes the new H
 * into H_dev, in work enqueued on `stream` or finished before it returns, and returns 0; any other
 * value ends the solve with CQ_ERR_CALLBACK.  It may call this library's matrix entry points on
 * the solver's system (cq_matrix_sum and the like), not the cq_lnv_* entry points of this solver.
 * fn = NULL switches the coupling off (the default). */
typedef int (*cq_h_rebuild_fn)(void* user, const double* K_dev, double* H_dev, int64_t length, void* stream);
int cq_lnv_set_h_rebuild(cq_lnv* s, cq_h_rebuild_fn fn, void* user);

/* Reduction log (tracing): with enable = 1 every later trace and product trace of the chain
 * (matrix_trace / matrix_product_trace values, in call order) is recorded.  Each call returns
 * the values recorded so far (*n of them, at most cap copied to out), clears the log and sets
 * the new state.  Two chains that take the same steps log the same sequence, so the first
 * differing entry locates the first differing step. */
int cq_lnv_reduction_log(cq_lnv* s, int enable, double* out, int64_t cap, int64_t* n);

/* Iteration record of the last cq_lnv_solve (the reference's list of Pulay residuals and
 * energies, PulayR / PulayE, DMMinModule.f90:289-294, with its per-iteration printout,
 * DMMinModule.f90:539-541 and 1000-1002): one entry per earlyDM and lateDM iteration, five
 * doubles each -- the residual g, the band energy 2 Tr(K H), the number of block products
 * run by the solve so far, 1.0 if the iteration's products were split-precision (0.0 for
 * FP64), and the host seconds since the solve started (taken once the residual has been read
 * from the device).  *n = entries recorded (at most 65536), at most cap of them copied to out
 * (5 * cap doubles).  Cleared when the next solve starts. */
int cq_lnv_residual_history(cq_lnv* s, double* out, int64_t cap, int64_t* n);

/* ------------------------------------------------------------------------ */
/* Serving loop: continuous batching of independent density-matrix solves    */
/* (no counterpart in the reference, which solves one system per run).       */
/* ------------------------------------------------------------------------ */
/*
 * A server owns `n_slots` worker threads, each with its own non-blocking CUDA stream on the
 * device current at creation.  Submitted requests queue in arrival order; a free slot admits the
 * first queued request whose memory estimate fits into what `hbm_budget` leaves after the
 * admitted ones (a request overtaken `max_bypass` times blocks later ones until it fits; one that
 * exceeds the whole budget runs alone).  An admitted request keeps its geometry, indices, S, H,
 * L and every temporary on the device from index build to result: S and H come from the
 * synthetic generators of cq_generate_SH with the request's seed, then cq_lnv_solve runs with
 * the server's parameters (`mixed` per request).  Solves of different slots overlap on the
 * device; each result is bit-identical to the same solve run alone (all reductions are exact
 * and every kernel is deterministic).  Times are seconds since the server was created.
 */
typedef struct {
  int n_slots;             /* concurrent solves (1..64) */
  int64_t hbm_budget;      /* bytes the admitted requests' estimates may hold together */
  int max_bypass;          /* times a queued request may be overtaken by later, smaller ones */
  int blocking_sync;       /* host waits sleep (CQ_OPT_BLOCKING_SYNC) */
  int dry_run;             /* 1: no device work; a request holds its slot and budget for
                              dry_run_seconds (scheduler tests without a GPU) */
  double dry_run_seconds;
  cq_lnv_params lnv;       /* solver parameters of every request (lnv.mixed is overridden) */
  int batch_products;      /* 1: the FP64 products of the slots' solves are gathered and run together,
                              one persistent launch per gathering (cq_mat_mult_batch; CUDA graphs of
                              the LNV calls off); a product waits at most batch_window_us for others */
  double batch_window_us;
} cq_server_config;

typedef struct {
  int n_atoms;
  const double* coords;    /* 3*n_atoms, bohr (copied at submit) */
  const double* cell;      /* 3 orthorhombic cell lengths */
  const int* nsf;          /* n_atoms block sizes */
  double rs, rh, rl, rt;   /* S, H, L and T ranges; the chain's other ranges follow (dimens_module) */
  double ne_spin;          /* electrons per spin channel */
  uint64_t seed;           /* S/H generator seed */
  int mixed;               /* 1: split-precision phase first (cq_lnv_params.mixed) */
  double t_arrival;        /* arrival time on the server clock (< 0: the time of submission) */
} cq_request;

typedef struct {
  int64_t id;
  int status;              /* CQ_OK or the CQ_ERR_* code of the failed solve */
  int n_atoms, converged, mixed, slot;
  double energy, electrons, residual;
  int64_t n_products, flops, n_products_mixed, flops_mixed;
  double t_arrival, t_admit, t_done;    /* latency = t_done - t_arrival */
  int64_t bytes_estimate;  /* admission estimate */
  int64_t bytes_peak;      /* device bytes the solve actually held at its peak */
  char message[128];       /* error message when status != CQ_OK */
  int split_restarts;      /* cq_lnv_result.split_restarts of the solve */
} cq_request_result;

typedef struct cq_server cq_server;
int cq_server_config_default(cq_server_config* c);
int cq_server_create(const cq_server_config* c, cq_server** out);
/* Queue a request; *id identifies its result.  Returns immediately. */
int cq_server_submit(cq_server* s, const cq_request* r, int64_t* id);
/* Wait up to timeout_s (< 0: forever) for the result of `id` and remove it from the server;
 * CQ_ERR_TIMEOUT if it is not finished by then. */
int cq_server_wait(cq_server* s, int64_t id, double timeout_s, cq_request_result* out);
/* Seconds on the server clock. */
int cq_server_now(cq_server* s, double* t);
/* Memory estimate the admission uses for a request (bytes). */
int cq_request_estimate(const cq_request* r, int64_t* bytes);
/* Stop accepting work, finish what is queued or running, join the workers. */
int cq_server_destroy(cq_server* s);

#ifdef __cplusplus
}
#endif
#endif /* CQ_B200_H */
