/*
 * bdc_b200.h -- C ABI of the B200 Blahut-Arimoto (BA) engine for the binary
 * deletion channel BDC_{n,k}: inputs are the 2^n binary strings of length n,
 * outputs the 2^k strings of length k, W(y|x) = N(x,y) / C(n,k) with N(x,y)
 * the number of occurrences of y as a subsequence of x.
 *
 * Plain C types only (no torch, no C++).  Every function returns a
 * bdc_status; on failure bdc_last_error() gives a one-line reason.  Nothing
 * calls exit().  Every call on a handle makes the handle's device current on
 * the calling thread.
 *
 * Layouts (identical to the reference, Pintz45/BDC-Upper-Bounds-GPU):
 *   p[R]       probability of EACH string of an orbit, one entry per canonical
 *              representative in ascending order (backend/main_BAA.cu:46-64);
 *              R = number of orbits of {id, reverse, complement, rev-compl}
 *   ln q[2^{k-1}]  ln of the output marginal, indexed by the representative's
 *              value; non-representative slots and q == 0 hold 0
 *              (backend/BAA.cu:649-652, 573-580)
 *   cache_n_k  binary uint32 little endian, 2^{n+k} entries, index (x<<k)|y
 *              (backend/cache_io.h:7-44)
 *   dist_n_k.txt   one "%.17g" probability per line, same order as p
 *              (backend/main_BAA.cu:84-91, 113-119)
 */
#ifndef BDC_B200_H
#define BDC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    BDC_OK = 0,
    BDC_ERR_ARG = 1,          /* bad argument: NULL, size mismatch, n/k out of range */
    BDC_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    BDC_ERR_IO = 3,           /* cache or distribution file missing, short or malformed */
    BDC_ERR_NOMEM = 4,        /* the device has too little free memory */
    BDC_ERR_STATE = 5,        /* call out of order (no handle loaded, no p set) */
    BDC_ERR_UNSUPPORTED = 6,  /* (n,k) outside what this build supports */
    BDC_ERR_NUMERIC = 7       /* non-finite input or result */
} bdc_status;

typedef enum {
    BDC_ENGINE_AUTO = 0,      /* the fastest engine that supports (n,k) */
    BDC_ENGINE_COUNT = 1,     /* split-identity count path: q pass + D pass per iteration */
    BDC_ENGINE_FACTORED = 2,  /* Kronecker-factored passes (FP64 matrix products) */
    BDC_ENGINE_COUNT_FP32C = 3 /* the count path with its q and D sums in compensated FP32
                                  (two-float accumulators, exact FP32 counts: n <= 26);
                                  FP64 for the q fold, the update and the bound's max.
                                  Opt-in: slower than the FP64 engines on a B200 */
} bdc_engine;

typedef struct {
    int engine;               /* bdc_engine */
    int device;               /* CUDA device ordinal */
    const char* cache_dir;    /* directory holding cache_n_k files (the reference's
                                 transition_counts/); NULL builds the half tables on
                                 the device with the GPU generator */
    int verbose;              /* print load/progress lines to stdout */
} bdc_options;

typedef struct {
    int64_t iters;            /* iterations done by this call */
    int64_t total_iters;      /* iterations since the distribution was set */
    double mx;                /* max_x log2 p'(x) - log2 p(x) of the last iteration (bits) */
    double upper_bound;       /* max_x D(x) of the last iteration's D pass (bits): C <= this */
    double rate;              /* sum_x p(x) D(x) of that iterate (bits) = I(p;W) */
    double lse;               /* log2 sum_x p(x) 2^{D(x)} of that iterate (bits) */
    double best_upper_bound;  /* min of max_x D(x) over every iterate evaluated since the
                                 distribution was set (bits): C <= this */
    double best_rate;         /* max of I(p;W) over those iterates (bits): this <= C */
    int converged;            /* bdc_iterate: 1 when the last mx < a (the loop of
                                 main_BAA.cu:73 ends); bdc_accelerate: 1 when
                                 best_upper_bound - best_rate < gap */
} bdc_stats;

typedef struct bdc_handle* bdc_handle_t;

void bdc_default_options(bdc_options* opts);
const char* bdc_last_error(void);
const char* bdc_version(void);

/* ---------------------------------------------------------------- handle
 * Replaces load_cache (backend/BAA.cu:183-188, decl. BAA.cuh:29) and its parts
 * load_gpu_cache / compute_normalizers / load_log_counts (BAA.cu:27-178): the
 * handle owns every device buffer, for one (n,k), until bdc_destroy.
 * 1 <= k <= n <= 32 for the count engine; the factored engine needs k < n. */
bdc_status bdc_create(int n, int k, const bdc_options* opts, bdc_handle_t* out);
bdc_status bdc_destroy(bdc_handle_t h);
bdc_status bdc_info(bdc_handle_t h, int* n, int* k, int64_t* num_reps, int* engine);

/* canonical representatives, ascending (backend/main_BAA.cu:46-50) */
bdc_status bdc_get_reps(bdc_handle_t h, uint32_t* reps, int64_t num_reps);

/* starting distribution (backend/main_BAA.cu:59-65); not renormalised,
 * like the reference.  Zero entries follow the reference's ln 0 = 0 rule. */
bdc_status bdc_set_p(bdc_handle_t h, const double* p, int64_t num_reps);
bdc_status bdc_set_p_uniform(bdc_handle_t h);           /* p = 1 / 2^n */
bdc_status bdc_get_p(bdc_handle_t h, double* p, int64_t num_reps);
/* device-pointer forms (the caller's memory on the handle's device) */
bdc_status bdc_set_p_device(bdc_handle_t h, const double* p_dev, int64_t num_reps);
bdc_status bdc_get_p_device(bdc_handle_t h, double* p_dev, int64_t num_reps);

/* The BA loop body (backend/main_BAA.cu:73-109 with baa_iteration,
 * BAA.cu:590-639 and compute_max_deviation, BAA.cu:916-946): runs iterations
 * until mx < a or max_iters iterations, all on the device.  stats may be NULL. */
bdc_status bdc_iterate(bdc_handle_t h, int64_t max_iters, double a, bdc_stats* stats);

/* Error of the last reported bound (no counterpart in the reference): for a
 * BDC_ENGINE_COUNT_FP32C handle, re-evaluates q and D in FP64 at the iterate
 * the last bdc_iterate's D pass used and returns |upper_bound - FP64 value|
 * and |rate - FP64 value| in bits; 0 and 0 for the FP64 engines.  Needs at
 * least one iteration since the distribution was set (BDC_ERR_STATE). */
bdc_status bdc_bound_error(bdc_handle_t h, double* upper_bound_err_bits, double* rate_err_bits);

/* Accelerated BA (no counterpart in the reference, whose loop is plain BA,
 * backend/main_BAA.cu:73-109): Nesterov-accelerated exponentiated gradient
 * driven by the adjoint of I(p;W).  Over the probabilities of the strings
 * the gradient is dI/dp(x) = D(x) - 1, and the mirror step of length eta is
 * ln p' = ln y + eta D(y) - ln Z (eta = 1, y = p: the BA update).  Each step
 * evaluates D at the extrapolated point y_t = x_t + beta_t (x_t - x_{t-1})
 * in ln p (beta_t = t / (t + 3)) and steps with eta = 1.5; when I(y_t) falls
 * below the last accepted I, the step is discarded and the momentum restarts
 * from x_t.  All on the device (8 steps per CUDA graph, the decisions are
 * kernels).  Every evaluated point gives a valid bracket, so best_rate <= C
 * <= best_upper_bound holds throughout.  Runs until best_upper_bound -
 * best_rate < gap_bits or max_evals evaluations; stats->iters = evaluations.
 * With 0 < gap_bits < 1e-4 (and n <= 26) the momentum phase stops at a
 * 1e-4-bit bracket and the support phases of bdc_solve finish: BA
 * restricted to the inputs that can carry mass, Newton on that support, and
 * a full-space evaluation proving that no other input can (the momentum
 * phase alone converges sublinearly on the small-mass members of the
 * support).  gap_bits <= 0 runs the momentum loop for max_evals.  The
 * handle's iterate is left at the final point.  Factored engine only;
 * BDC_ACCEL_STEP overrides eta (0 < eta <= 4). */
bdc_status bdc_accelerate(bdc_handle_t h, int64_t max_evals, double gap_bits, bdc_stats* stats);

/* The mutual-information functional and its adjoint (no counterpart in the
 * reference).  Forward: I(p;W) in nats for p (host, one entry per
 * representative, not necessarily normalised; NULL: the current iterate),
 * which becomes the current iterate.  Backward: grad[i] = dI/dp_i in nats for
 * the current iterate, where p_i moves the probability of every string of
 * orbit i together: grad[i] = |O_i| (D(x_i) - 1). */
bdc_status bdc_mi_forward(bdc_handle_t h, const double* p, int64_t num_reps, double* I_nats);
bdc_status bdc_mi_backward(bdc_handle_t h, double* grad, int64_t num_reps);
/* The same gradient written to device memory the caller owns (on the
 * handle's device), for optimisers that keep their iterate on the GPU:
 * bdc_set_p_device, bdc_mi_forward(h, NULL, ...), bdc_mi_backward_device.
 * Returns when grad_dev is written. */
bdc_status bdc_mi_backward_device(bdc_handle_t h, double* grad_dev, int64_t num_reps);

/* Certified solver (no counterpart in the reference, which runs plain BA
 * until max_x log2 p'/p < a, backend/main_BAA.cu:73).  Anderson-accelerated
 * BA on all inputs, then BA restricted to the inputs that can carry mass,
 * then a full evaluation that proves no other input can (and widens the set
 * if one could).  Every reported number is evaluated exactly at its point:
 * best_rate = I(p;W) <= C <= best_upper_bound = max_x D(x).  Runs until the
 * bracket is below gap_bits or max_evals full-space BA evaluations; the
 * handle's iterate becomes the final point (entries that are zero there stay
 * zero under later iterations).  stats->iters = full-space evaluations,
 * stats->mx = the bracket in bits, converged = bracket < gap_bits.  Factored
 * engine, n <= 26. */
bdc_status bdc_solve(bdc_handle_t h, double gap_bits, int64_t max_evals, bdc_stats* stats);

/* Sharded BA (no counterpart in the reference, which runs one (n,k) on one
 * GPU): rank r of a group owns the representatives [rep_begin, rep_end) of a
 * count-engine handle (every rank holds the whole problem and sets the same
 * distribution) and touches p only there.  One iteration:
 *   bdc_shard_q(acc)             partial q sums, acc[y] for all 2^k raw y
 *   -- the caller sums acc over the ranks (an all-reduce) --
 *   bdc_shard_set_q(acc)         ln q from the summed sums
 *   bdc_shard_update_begin(st)   D and logW on the shard; st = {s = max logW,
 *                                Z = sum |O| exp(logW - s), max D (nats),
 *                                sum |O| p D (nats), input-zero flag}
 *   -- the caller forms S = max s, Z_all = sum Z exp(s - S) over the ranks,
 *      the bound max D and the rate sum --
 *   bdc_shard_update_end(ln Z_all + S - s, &mx)   p' on the shard, local mx
 *   -- the caller takes the max of mx over the ranks (the stopping rule) --
 * bdc_b200.sharded runs this loop over torch.distributed.  After a sharded
 * iteration the handle's own last bound, rate and mx (bdc_iterate's stats)
 * describe its shard, not the whole problem; the loop's combined values are
 * the sharded problem's.  The handle's best-bound trackers are not touched. */
bdc_status bdc_shard_q(bdc_handle_t h, int64_t rep_begin, int64_t rep_end, double* acc, int64_t ny);
bdc_status bdc_shard_set_q(bdc_handle_t h, const double* acc, int64_t ny);
bdc_status bdc_shard_update_begin(bdc_handle_t h, int64_t rep_begin, int64_t rep_end, double* stats5);
bdc_status bdc_shard_update_end(bdc_handle_t h, int64_t rep_begin, int64_t rep_end, double log_z, double* mx);

/* The factored engine with its rows sharded over several GPUs (no
 * counterpart in the reference, which runs one (n,k) on one GPU).  Rank r of
 * `world` holds a window of whole rows x_hi (about R / world representatives,
 * a contiguous range of the ascending list): the dense iterate, h(x) and the
 * G product exist only for those rows.  Every rank sets the same
 * distribution (bdc_set_p with the full vector).  One iteration:
 *   bdc_fshard_q(acc)              partial q sums of the held rows, 2^k values
 *   -- the caller sums acc over the ranks (an all-reduce) --
 *   bdc_fshard_d(acc, part5)       ln q, the D side and G with the update on the
 *                                  held rows; part5 = [max D, sum |O| e,
 *                                  max logW, sum |O| p D, input-zero flag]
 *   -- the caller combines part5 over the ranks: max, sum, max, sum, max --
 *   bdc_fshard_finish(part5, a, stats)   ln Z, mx, the bound and the stop test,
 *                                  identical on every rank (stats->converged: mx < a)
 * A sharded handle refuses the single-GPU calls (bdc_iterate, bdc_get_p, ...);
 * bdc_fshard_get_p returns p of its own representatives.  bdc_b200.sharded
 * runs this loop over torch.distributed. */
bdc_status bdc_create_sharded(int n, int k, const bdc_options* opts, int rank, int world, bdc_handle_t* out);
bdc_status bdc_fshard_range(bdc_handle_t h, int* row0, int* rows, int64_t* rep_begin, int64_t* rep_end);
bdc_status bdc_fshard_q(bdc_handle_t h, double* acc, int64_t ny);
bdc_status bdc_fshard_d(bdc_handle_t h, const double* acc, int64_t ny, double* part5);
bdc_status bdc_fshard_finish(bdc_handle_t h, const double* part5, double a, bdc_stats* stats);
bdc_status bdc_fshard_get_p(bdc_handle_t h, double* p, int64_t count);

/* Batches (no counterpart in the reference, which runs one (n,k) per
 * process): many handles -- different (n,k) and starting distributions --
 * iterated together from one captured CUDA graph with one branch per handle.
 * bdc_batch_iterate runs the BA loop of every handle until each one's mx < a
 * (it then idles) or max_iters; stats (may be NULL) receives one entry per
 * handle, in the order given.  The handles stay owned by the caller and must
 * outlive the batch; they must all be on one device. */
typedef struct bdc_batch* bdc_batch_t;
bdc_status bdc_batch_create(bdc_handle_t* handles, int count, bdc_batch_t* out);
bdc_status bdc_batch_iterate(bdc_batch_t batch, int64_t max_iters, double a, bdc_stats* stats);
bdc_status bdc_batch_destroy(bdc_batch_t batch);
/* Queue the batch's work on a caller's cudaStream_t (NULL: the batch's own
 * stream); bdc_batch_iterate still returns only when that work is done. */
bdc_status bdc_batch_set_stream(bdc_batch_t batch, void* stream);
/* The accelerated loop of bdc_accelerate for every handle of the batch (all
 * factored engine), 8 steps of each per replay of one captured graph, each
 * instance stopping on its own bracket (best_upper_bound - best_rate <
 * gap_bits) or after max_evals evaluations.  seconds (may be NULL) receives
 * per instance the device time from the start of the call until its bracket
 * fell below gap_bits (CUDA events on the launch stream, resolution one graph
 * replay), -1 when it did not.  With 0 < gap_bits < 1e-4 the batched
 * momentum phase runs to a 1e-4-bit bracket and then each instance's support
 * phases finish it, one instance after another; its time is then its
 * momentum phase in the batch plus its own support phases. */
bdc_status bdc_batch_accelerate(bdc_batch_t batch, int64_t max_evals, double gap_bits, bdc_stats* stats,
                                double* seconds);

/* One reference-shaped iteration with host vectors: p_in -> p_out, like
 * baa_iteration (BAA.cu:590-639, decl. BAA.cuh:295); p_out may equal p_in. */
bdc_status bdc_baa_iteration(bdc_handle_t h, const double* p_in, double* p_out, int64_t num_reps);

/* compute_all_log_D (BAA.cu:642-724, decl. BAA.cuh:314): ln q of the current p */
bdc_status bdc_log_q(bdc_handle_t h, double* lnq, int64_t nq);
/* compute_all_log_W (BAA.cu:727-814, decl. BAA.cuh:342): ln p + D for the
 * current p and a caller-given ln q (NULL: ln q of the current p) */
bdc_status bdc_log_w(bdc_handle_t h, const double* lnq, double* logw, int64_t num_reps);
/* compute_KL_kernel (BAA.cu:533-571, decl. BAA.cuh:266): D(x) in nats for a
 * caller-given ln q (NULL: ln q of the current p) */
bdc_status bdc_divergence(bdc_handle_t h, const double* lnq, double* d, int64_t num_reps);
/* compute_rate (BAA.cu:836-913, decl. BAA.cuh:348): sum |O| p D in nats with
 * ln q of the current p */
bdc_status bdc_rate(bdc_handle_t h, double* rate_nats);
/* compute_max_deviation (BAA.cu:916-946, decl. BAA.cuh:361) on host vectors */
bdc_status bdc_max_deviation(bdc_handle_t h, const double* p, const double* p_before,
                             int64_t num_reps, double* mx);

/* exact counts N(x,y) by the split identity (total_transitions, BAA.cu:340-395)
 * for npairs host pairs; out[i] = N(xs[i], ys[i]) */
bdc_status bdc_counts(bdc_handle_t h, const uint32_t* xs, const uint32_t* ys, int64_t npairs,
                      uint32_t* out);

/* ----------------------------------------------------------- measurement
 * Algorithmic work of one pass over the channel matrix: nonzero_pairs =
 * sum over representatives x of the number of distinct length-k
 * subsequences of x (the pairs the reference enumerates, BAA.cu:460), and
 * split_terms = number of split points j of total_transitions (BAA.cu:355). */
bdc_status bdc_work(bdc_handle_t h, int64_t* nonzero_pairs, int* split_terms);

typedef struct {
    double ms_q;        /* q pass (count engine) or q-side products (factored) */
    double ms_fold;     /* orbit fold of q and ln q */
    double ms_d;        /* D pass (count engine) or D-side products + update (factored) */
    double ms_update;   /* normalisation, mx and stop test */
    double ms_iter;     /* whole iteration */
    double ms_main;     /* the dominant kernel alone: the D pass (count engine) or
                           the fused D-side product G = LA * RB (factored engine) */
    double work_main;   /* its algorithmic work per launch: split-term multiply-adds
                           over the nonzero pairs (count) or FP64 flops (factored) */
    int launches;       /* kernel launches per iteration */
    int iters;          /* iterations averaged */
    int main_kind;      /* the dominant kernel: 0 the count D pass, 1 G on the FP64
                           tensor path (mma.sync), 2 G on the int8 tensor cores */
    double bytes_main;  /* its algorithmic device-memory bytes per launch: the
                           update's 40 bytes per representative (read h, ln p, p;
                           write ln p, p) for G, 0 for the count D pass */
} bdc_profile_t;

/* Runs `iters` iterations (a = -inf, so none stops early) with CUDA events
 * around each pass on the handle's stream; averages in milliseconds.  The
 * iterate advances like bdc_iterate. */
bdc_status bdc_profile(bdc_handle_t h, int iters, bdc_profile_t* out);

/* Run the handle's work on a caller-owned cudaStream_t (NULL: the handle's
 * own stream), e.g. to order it with a framework's stream or to time it with
 * events recorded on that stream. */
bdc_status bdc_set_stream(bdc_handle_t h, void* cuda_stream);

/* Device throughput probe: kind 0 = int32 multiply-add (IMAD), 1 = FP64 FMA,
 * 2 = FP32 FMA, 3 = FP64 tensor-core multiply-add (mma.sync m8n8k4).  Runs a register-resident chain kernel on `device` for about
 * `ms` milliseconds and returns operations per second (one multiply-add = 1
 * operation).  Used as the measured denominator of roofline fractions. */
bdc_status bdc_peak_probe(int device, int kind, double ms, double* ops_per_s);

/* Allocation-free variant of bdc_max_deviation (no counterpart in the
 * reference): max_i log2 p[i] - log2 p_before[i] over device arrays the
 * caller owns, written to the device double *mx_dev, queued on cuda_stream
 * (NULL: the legacy default stream).  For callers that cannot allocate
 * device memory (their own pool or arena owns it all, or an allocator call
 * is not allowed where they run): no handle, no cudaMalloc/cudaFree.  The
 * reduction's block partials live in one fixed 128 KB array per device,
 * shared by every call: num_reps <= 2^27 (else BDC_ERR_ARG), calls whose
 * kernels overlap on the GPU race, and the first call on a device (which
 * looks up the array's address) should come before any stream capture. */
bdc_status bdc_max_deviation_noalloc(const double* p_dev, const double* p_before_dev, int64_t num_reps,
                                     double* mx_dev, void* cuda_stream);

/* ------------------------------------------------------- cache generator
 * The table cache_{n,k} of generate_bit_transition_cache.cpp:46-77, computed on
 * the device: out holds 2^{n+k} uint32, index (x << k) | y.  n + k <= 34. */
bdc_status bdc_generate_cache(int n, int k, int device, uint32_t* out);

/* ------------------------------------------------------------ file formats */
/* read a cache_n_k file (cache_io.h:29-44): exactly 2^{n+k} entries */
bdc_status bdc_read_cache_file(const char* path, int n, int k, uint32_t* out);
/* write a cache_n_k file (cache_io.h:17-26) */
bdc_status bdc_write_cache_file(const char* path, int n, int k, const uint32_t* data);
/* read a dist file (main_BAA.cu:3-18); *count gets the number of values.
 * With out == NULL only counts. */
bdc_status bdc_read_dist_file(const char* path, double* out, int64_t cap, int64_t* count);
/* write a dist file with "%.17g\n" per value, via a temporary file and rename */
bdc_status bdc_write_dist_file(const char* path, const double* p, int64_t count);

#ifdef __cplusplus
}
#endif

#endif /* BDC_B200_H */
