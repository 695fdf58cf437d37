/*
 * tspb.h - C ABI of libtspb.so, the B200 (sm_100a) kernels behind the memetic-GA
 * hot path of lucasgaldinos/tsp_gpu_clean.
 *
 * Conventions (every entry point):
 *   - plain device pointers and sizes; no framework types;
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream);
 *   - work is enqueued asynchronously on `stream`; the return value is a host-side
 *     status (TSPB_OK or a TSPB_ERR_* code) covering argument checks and the launch;
 *   - per-item device-side failures (a tour that is not a permutation, an index out
 *     of range) are written to the optional `status` device array, one int32 per
 *     item, 0 meaning success; the item is then left unchanged;
 *   - node ids are int32 in [0, dim); distance matrices are int32, row-major with
 *     `dist_stride` elements per row; coordinates are float64 (x, y) pairs.
 *
 * Reference file:line citations are relative to the reference project root.
 */
#ifndef TSPB_H
#define TSPB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TSPB_OK 0
#define TSPB_ERR_ARG 1            /* bad size, null pointer, unknown mode */
#define TSPB_ERR_CUDA 2           /* a CUDA launch or query failed */
#define TSPB_ERR_NOT_PERMUTATION 3 /* an input tour repeats or misses a node */
#define TSPB_ERR_RANGE 4          /* a value exceeds what the kernel's integer math covers */
#define TSPB_ERR_UNSUPPORTED 5    /* configuration outside the kernels' scope */
#define TSPB_ERR_WORKSPACE 6      /* caller workspace smaller than tspb_*_workspace_bytes */
#define TSPB_ERR_BUDGET 7         /* a tour hit the device watchdog before converging */
#define TSPB_ERR_DEVICE_MEMORY 8  /* the device could not provide memory the library itself holds */

#define TSPB_MODE_BEST 0       /* steepest move per pass; also the "batch" mode */
#define TSPB_MODE_FIRST 1      /* first improving move in scan order */
#define TSPB_MODE_MULTI_MOVE 2 /* every disjoint improving move, steepest first */
/* OR-ed into a 2-opt mode: the distances are symmetric (d(a, b) == d(b, a) for every pair),
 * as EUC_2D from coordinates is. After a move that reverses a window wider than the CTA,
 * the candidate scan then takes each reversed node's new out-edge from its old
 * predecessor's (the same edge) and reads only the two new edges from the distance source.
 * Without it every out-edge of the reversed window is read again, which is exact for
 * asymmetric matrices too. Launches that rebuild distances from coordinates (no matrix)
 * are symmetric without it. Results are the same either way on symmetric distances. */
#define TSPB_MODE_SYMMETRIC 0x100

/* Library version and build facts. */
int tspb_version(void);

/* Human-readable text for a TSPB_* status code (static storage). */
const char* tspb_status_string(int status);

/*
 * Device watchdog of the local-search kernels (2-opt in every mode, the batch 2-opt,
 * Or-opt, 3-opt): a tour that has not converged after `cycles` SM clock cycles ends with
 * TSPB_ERR_BUDGET, its tour left a valid permutation (the moves applied so far) and its
 * stats counting the passes run. Applies to launches made after the call, process-wide;
 * a launch captured in a CUDA graph keeps the budget it was captured with. cycles <= 0
 * restores the default (2^36 cycles, about 35 s at 1.9 GHz). Returns the previous budget.
 * No counterpart in the reference (its loops run on the host and stop on max_iterations).
 */
int64_t tspb_set_watchdog_cycles(int64_t cycles);

/* Bytes of global scratch `tspb_two_opt` needs for this shape (0 when none). */
size_t tspb_two_opt_workspace_bytes(int32_t num_tours, int32_t n, int32_t k, int32_t mode, int32_t block_threads);

/*
 * Batched 2-opt local search, one CTA per tour, in place on `tours` (num_tours x n).
 * Replaces: LocalSearchCPUTourTwoOpt._refine / improve_batch
 *   (src/algorithms/strategies/local_search/two_opt.py:565-628) with the pair order of
 *   _pair_blocks (:303-367), the gains of _pair_deltas (:204-261) and the acceptance
 *   rules _step_best (:386-440), _step_first (:442-489), _step_multi_move (:491-563);
 *   and the GPU launch loop of LocalSearchGPUTourTwoOpt._improve_grid (:831-899).
 * Cyclic TSP topology. `cand` (n x k, k-NN table) selects candidate mode; NULL selects
 * the exhaustive scan. `cand_dist` (n x k, optional) holds d(a, cand[a][r]).
 * Candidate best/first run the rescan kernel (block sizes 64, 128, 256 or 512) unless
 * `rev_off`/`rev_idx` (from tspb_candidate_reverse_index) are given without
 * `cand_packed`, which selects the cached kernel: per-row keys and pair counts kept
 * exactly across passes and refreshed only where a reversal can change them.
 * `cand_packed` (optional, from tspb_candidate_pack) lets the rescan kernel read id and
 * distance in one word; given together with `rev_off`/`rev_idx`, first mode restarts
 * incrementally: after a move with window [bi, bj] a pass evaluates only the entries of
 * rows before bi whose candidate lies in the window, then scans from row bi (the other
 * entries before bi cannot have changed). Results and stats[0..2] are the same either way.
 * Distances come from `dist` when non-NULL, else are rebuilt from `coords` in FP64
 * with TSPLIB EUC_2D rounding. `max_iterations` bounds the passes per tour.
 * `stats` (optional, num_tours x 4 int64): passes, pairs evaluated by the reference
 * scan (oracle-equivalent deltas), reversals applied, gains computed by the kernel.
 */
int tspb_two_opt(int32_t* tours, int32_t num_tours, int32_t n,
                 const int32_t* dist, int64_t dist_stride, const double* coords,
                 const int32_t* cand, const int32_t* cand_dist,
                 const int32_t* rev_off, const int32_t* rev_idx, const uint32_t* cand_packed, int32_t k,
                 int32_t mode, int64_t max_iterations, int32_t block_threads,
                 int64_t* stats, int32_t* status,
                 void* workspace, size_t workspace_bytes, void* stream);

/*
 * tspb_two_opt that becomes a no-op on the device when *skip (device int32) is non-zero
 * at launch time: tours, stats and status are then left untouched. Lets a captured CUDA
 * graph of GA generations stop refining once the run's stop flag is set. No reference
 * counterpart (the reference loop stops on the host).
 */
int tspb_two_opt_gated(const int32_t* skip, int32_t* tours, int32_t num_tours, int32_t n,
                       const int32_t* dist, int64_t dist_stride, const double* coords,
                       const int32_t* cand, const int32_t* cand_dist,
                       const int32_t* rev_off, const int32_t* rev_idx, const uint32_t* cand_packed, int32_t k,
                       int32_t mode, int64_t max_iterations, int32_t block_threads,
                       int64_t* stats, int32_t* status,
                       void* workspace, size_t workspace_bytes, void* stream);

/*
 * multi_move 2-opt (same kernel and results as tspb_two_opt with TSPB_MODE_MULTI_MOVE)
 * that allocates nothing: its scratch is a fixed TSPB_STATIC_SCRATCH_BYTES array compiled
 * into the library, which every GPU that loads the library holds until exit. No
 * counterpart in the reference. It is for callers that cannot call cudaMalloc, such as
 * code running inside a host callback or a latency-critical loop that must stay off the
 * allocator, or a plugin host that owns all device memory and passes in only the input
 * and output buffers. The caller still provides tours, distances, candidates and the
 * optional stats/status buffers.
 *   - Returns TSPB_ERR_WORKSPACE when the shape needs more scratch than the array holds
 *     (tspb_two_opt_workspace_bytes(num_tours, n, k, TSPB_MODE_MULTI_MOVE, threads) >
 *     TSPB_STATIC_SCRATCH_BYTES); split the batch into smaller calls then.
 *   - The first call on a device looks up the array's device address (set-up, once per
 *     device, with that device current); make that first call before any stream capture.
 *     Under lazy module loading (CUDA_MODULE_LOADING=LAZY, CUDA's default) that first call
 *     is also when the device reserves the array, so a caller that must not allocate later
 *     makes it during its own set-up. When the device cannot provide the array the call
 *     returns TSPB_ERR_DEVICE_MEMORY (other lookup failures: TSPB_ERR_CUDA) and clears the
 *     CUDA error it caused.
 *   - The address is kept per device with the identity of the context it belongs to; after
 *     a reset of the device's context (cudaDeviceReset, or the primary context released and
 *     created again) the next call looks it up again, reserving the array anew.
 *   - All calls share the array: calls whose kernels overlap on the GPU race on it and
 *     must be serialised by the caller.
 */
#define TSPB_STATIC_SCRATCH_BYTES (32u << 20)
int tspb_two_opt_multi_move_static(int32_t* tours, int32_t num_tours, int32_t n,
                                   const int32_t* dist, int64_t dist_stride, const double* coords,
                                   const int32_t* cand, const int32_t* cand_dist, int32_t k,
                                   int64_t max_iterations, int32_t block_threads,
                                   int64_t* stats, int32_t* status, void* stream);

/*
 * cand_dist[a*k + r] = d(a, cand[a*k + r]) for the n x k table (entries outside [0, n)
 * give 0). Replaces the D[a, c] gathers of _pair_deltas (two_opt.py:242) with a table
 * built once per instance.
 */
int tspb_candidate_distances(const int32_t* cand, int32_t n, int32_t k,
                             const int32_t* dist, int64_t dist_stride, const double* coords,
                             int32_t* cand_dist, void* stream);

/*
 * Reverse k-NN index in CSR form: for node c, rev_idx[rev_off[c] .. rev_off[c+1]) lists
 * the flat entries a*k + r with cand[a*k + r] == c (order within a list unspecified).
 * rev_off has n + 1 entries, rev_idx n*k, scratch n int32. No reference counterpart:
 * it serves the cached 2-opt kernel's refresh of gains whose second city moved.
 */
int tspb_candidate_reverse_index(const int32_t* cand, int32_t n, int32_t k, int32_t* rev_off,
                                 int32_t* rev_idx, int32_t* scratch, void* stream);

/*
 * packed[e] = cand[e] | cand_dist[e] << 16 for the n x k table; *overflow (device int)
 * becomes 1 when an id or distance does not fit 16 bits (the packed table must then not
 * be used). No reference counterpart: a layout of the k-NN table for the 2-opt scan.
 */
int tspb_candidate_pack(const int32_t* cand, const int32_t* cand_dist, int32_t n, int32_t k,
                        uint32_t* packed, int32_t* overflow, void* stream);

/*
 * Closed-tour cost per row (sum of n edges incl. the closing edge when return_to_depot),
 * written as float64. Replaces evaluate_tour_cpu
 *   (src/algorithms/strategies/evaluation/tour_cost.py:17-29) and tour_cost_kernel
 *   (src/algorithms/strategies/evaluation/kernels/tour_cost.cu:21-63).
 */
int tspb_tour_cost(const int32_t* tours, int32_t num_tours, int32_t n,
                   const int32_t* dist, int64_t dist_stride, const double* coords,
                   int32_t return_to_depot, double* costs, void* stream);

/*
 * Tournament selection: winners[p] = first argmin of fitness over cand[p*k .. p*k+k).
 * Replaces SelectionCPUTournament.select_batch
 *   (src/algorithms/strategies/selection/tournament_selection.py:98-128) and
 *   tournament_selection_kernel (.../selection/kernels/tournament_selection.cu:11-39).
 */
int tspb_tournament(const double* fitness, int32_t pop_size, const int32_t* cand,
                    int32_t num_parents, int32_t k, int32_t* winners, void* stream);

/* out[r, :] = src[rows[r], :] for r < num_rows (row gather of an int32 matrix). */
int tspb_gather_rows(const int32_t* src, int32_t src_rows, int32_t n, const int32_t* rows,
                     int32_t num_rows, int32_t* out, void* stream);

/* dst[rows[r], :] = src[r, :] for r < num_rows (rows outside [0, dst_rows) skipped).
 * Replaces the elite scatter-back `state.population[elite_indices] = improved`
 * (src/algorithms/pipeline_steps.py:183). */
int tspb_scatter_rows(const int32_t* src, int32_t num_rows, int32_t n, const int32_t* rows, int32_t* dst,
                      int32_t dst_rows, void* stream);

/*
 * PMX crossover of pairs (2q, 2q+1) sharing cuts (first[q], second[q]); the odd tail
 * row is copied. Open permutations (bounds [0, n)). Replaces
 *   CrossoverCPUPermPartiallyMapped._apply_pmx / crossover_batch
 *   (src/algorithms/strategies/crossover/pmx_crossover.py:49-105, 128-171) and
 *   pmx_crossover_kernel (.../crossover/kernels/pmx_crossover.cu:19-154).
 */
int tspb_pmx(const int32_t* parents, int32_t num_routes, int32_t n,
             const int32_t* cut_first, const int32_t* cut_second,
             int32_t* children, int32_t* status, void* stream);

/*
 * Order Crossover (OX) of pairs (2q, 2q+1) sharing cuts (first[q], second[q]); the odd
 * tail row is copied. Open permutations. The child keeps p1[c1..c2]; the free positions
 * c2+1, ..., n-1, 0, ..., c1-1 take p2's remaining genes in the order met reading p2 from
 * c2+1 (wrapping). Replaces CrossoverCPUPermOrder._apply_ox / crossover_batch
 *   (src/algorithms/strategies/crossover/order_crossover.py:52-83, 127-168) and
 *   order_crossover_kernel (.../crossover/kernels/order_crossover.cu).
 * A parent that is not a permutation of 0..n-1 gives status[row] = TSPB_ERR_NOT_PERMUTATION
 * and the child is a copy of p1.
 */
int tspb_ox(const int32_t* parents, int32_t num_routes, int32_t n,
            const int32_t* cut_first, const int32_t* cut_second,
            int32_t* children, int32_t* status, void* stream);

/*
 * Swap mutation in place: positions pos1[r], pos2[r] of row r exchanged when u[r] < rate.
 * Replaces MutationCPUPermSwap.mutate_batch
 *   (src/algorithms/strategies/mutation/swap_mutation.py:65-99) and swap_mutation_kernel
 *   (.../mutation/kernels/swap_mutation.cu).
 */
int tspb_swap(int32_t* routes, int32_t num_routes, int32_t n, const double* u,
              double rate, const int32_t* pos1, const int32_t* pos2, void* stream);

/* Operators of the fused and batched generation. */
#define TSPB_XOVER_PMX 0
#define TSPB_XOVER_OX 1
#define TSPB_MUT_INVERSION 0
#define TSPB_MUT_SWAP 1

/*
 * Inversion mutation in place: row r reversed over [min(p1,p2), max(p1,p2)] when
 * u[r] < rate. Replaces MutationCPUPermInversion.mutate_batch
 *   (src/algorithms/strategies/mutation/inversion_mutation.py:65-99) and
 *   inversion_mutation_kernel (.../mutation/kernels/inversion_mutation.cu:11-44).
 */
int tspb_inversion(int32_t* routes, int32_t num_routes, int32_t n, const double* u,
                   double rate, const int32_t* pos1, const int32_t* pos2, void* stream);

/*
 * (mu + lambda) survival: order[0..keep) = indices of the `keep` smallest values of
 * fitness[0..count) by (fitness, index), i.e. a stable ascending sort. Replaces
 * GeneticAlgorithm._select_survivors_assessed for feasible tours
 *   (src/algorithms/metaheuristics/genetic_algorithm.py:618-706, lexsort :682-689).
 */
int tspb_stable_rank(const double* fitness, int32_t count, int32_t keep, int32_t* order, void* stream);

/*
 * GRASP nearest-neighbour initial population, one thread per row: row r starts from the
 * SplitMix64 stream seeded with seeds[r] and walks the k-NN table of `cand` (cand_rows x k).
 * `workspace` holds pop * (n + max_node + 1 + k) int32. Replaces
 *   InitializationCPUTourNearestNeighbor.initialize / _nearest_neighbor_row_cpu
 *   (src/algorithms/strategies/initialization/nearest_neighbor_init.py:31-132) and
 *   nearest_neighbor_init_kernel (.../initialization/kernels/nearest_neighbor_init.cu:10-111).
 */
int tspb_nn_init(const int32_t* customers, int32_t n, const int32_t* cand, int32_t cand_rows, int32_t k,
                 const uint64_t* seeds, int32_t pop, int32_t max_node, int32_t* workspace,
                 size_t workspace_bytes, int32_t* out, void* stream);

/*
 * Nearest-neighbour initial tours of many instances in one launch (customers 0..n-1 of
 * each job), thread per (job, row), each row computed exactly as tspb_nn_init computes it.
 * `jobs` is a device array; job j uses rows * (2 n + k) int32 of `workspace` from element
 * ws_offsets[j] (device int64 array); max_rows bounds every job's rows.
 */
typedef struct tspb_nn_job {
  int32_t n;              /* customers 0..n-1 */
  int32_t k;              /* k-NN entries per row of cand (0: uniform choices only) */
  const int32_t* cand;    /* n x k */
  const uint64_t* seeds;  /* [rows] SplitMix64 row seeds (draw_row_seeds) */
  int32_t* out;           /* rows x n */
  int32_t rows;
  int32_t pad;
} tspb_nn_job;
int tspb_nn_init_jobs(const tspb_nn_job* jobs, int32_t num_jobs, int32_t max_rows, int32_t* workspace,
                      const int64_t* ws_offsets, void* stream);
/* The same tours with every row's working arrays in shared memory (no workspace): max_n
 * and max_k bound every job's n and k; TSPB_ERR_UNSUPPORTED when 4 max_n + 2 max_k bytes
 * exceed 200 KB or max_n > 65535 (use tspb_nn_init_jobs then). */
int tspb_nn_init_jobs_smem(const tspb_nn_job* jobs, int32_t num_jobs, int32_t max_rows, int32_t max_n, int32_t max_k,
                           void* stream);

/*
 * Exhaustive steepest-descent 3-opt of open (cyclic TSP) tours in place, up to
 * max_iterations passes each, bit-identical to the reference's CPU 3-opt
 * (cpu_three_opt_best_move / cpu_three_opt_refine,
 * benchmark_scripts/experiments-and-examples/experiment-comparing-3opt-and-2opt/gpu_three_opt.py:143-277;
 * the GPU strategy LocalSearchGPUThreeOpt(mode="batch"/"naive") of the same file). Distances
 * from `dist` (n x dist_stride) or rebuilt from EUC_2D `coords`. One CTA per tour, `threads`
 * 128, 256 or 512; n <= 4096 (one pass is n^3/6 triples). For n above 220 each CTA needs n*n int32 of `workspace`
 * (tspb_three_opt_workspace_bytes); fewer CTAs are launched when the workspace holds fewer
 * tours (TSPB_ERR_WORKSPACE when it holds none). stats (optional): [tours][3] passes, moves,
 * (triple, case) candidates evaluated.
 */
int tspb_three_opt(int32_t* tours, int32_t num_tours, int32_t n, const int32_t* dist, int64_t dist_stride,
                   const double* coords, int64_t max_iterations, int32_t threads, int32_t* workspace,
                   size_t workspace_bytes, int32_t* status, int64_t* stats, void* stream);
int tspb_three_opt_workspace_bytes(int32_t n, int32_t ctas, size_t* bytes);

/*
 * 3-opt with the rules of the reference's grid kernels, for the two parts of its 3-opt
 * that only its CUDA kernels define (benchmark_scripts/experiments-and-examples/
 * experiment-comparing-3opt-and-2opt/kernels/three_opt_common.cuh:155-447,
 * three_opt_batch.cu, three_opt_multi_move.cu; driven by LocalSearchGPUThreeOpt._improve_grid,
 * gpu_three_opt.py:452-537):
 *   - k > 0: the candidate-pruned scan (cand: n x k sorted k-NN table, cand_dist its
 *     distances; inner_k <= 0 means k), one move per pass (multi_move = 0) or multi_move;
 *   - k == 0: the exhaustive scan, multi_move only (one-move exhaustive passes are
 *     tspb_three_opt, which follows the reference's CPU 3-opt).
 * The moves are those of the reference's kernel launched with
 * tspb_three_opt_grid_threads(threads_per_block, n) threads per tour (its
 * prev_power_of_2(min(threads_per_block, n)) clamped to 256). Open (cyclic TSP) tours of
 * every city, in place; up to max_iterations passes, stopping after a pass that applies
 * nothing. stats (optional, num_tours x 3): passes, moves applied, candidate moves
 * evaluated. Exhaustive n <= 4095; candidate n up to what 20 n bytes of shared memory hold.
 */
int tspb_three_opt_grid(int32_t* tours, int32_t num_tours, int32_t n, const int32_t* dist, int64_t dist_stride,
                        const double* coords, const int32_t* cand, const int32_t* cand_dist, int32_t k,
                        int32_t inner_k, int32_t multi_move, int32_t threads_per_block, int64_t max_iterations,
                        int32_t* status, int64_t* stats, void* stream);
int tspb_three_opt_grid_threads(int32_t threads_per_block, int32_t n);

/*
 * Candidate-list Or-opt of open (cyclic TSP) tours in place, best improvement, up to
 * max_iterations passes each. No reference counterpart (the reference's local search has
 * 2-opt and an experimental 3-opt); it widens the family with the reference's candidate
 * 2-opt conventions (src/algorithms/strategies/local_search/two_opt.py:347-367: k-NN
 * candidates, position 0 fixed, exact integer deltas, first move in scan order on ties).
 * A move relocates t[i .. i+L-1] (1 <= L <= max_segment <= 8, i >= 1) after a candidate c
 * of its first city (forward) or of its last city (reversed, L >= 2); the move applied is
 * the smallest negative delta, then the smallest key (((i-1)*max_segment + L-1)*k + r)*2 + o.
 * cand / cand_dist: n x k k-NN ids and d(a, cand) (1 <= k <= n-1, symmetric distances);
 * cand_packed (optional): the same as c | d << 16 words (tspb_candidate_pack, no overflow),
 * read four at a time when k % 4 == 0 and the table is 16-byte aligned;
 * distances from `dist` (n x dist_stride) or rebuilt from EUC_2D `coords`. One CTA per
 * tour (persistent), `threads` 128, 256 or 512, 16 n bytes of shared memory
 * (n <= tspb_or_opt_max_n()). n < 3: nothing to do. stats (optional): [tours][3] passes,
 * moves, valid entries evaluated.
 */
int tspb_or_opt(int32_t* tours, int32_t num_tours, int32_t n, const int32_t* dist, int64_t dist_stride,
                const double* coords, const int32_t* cand, const int32_t* cand_dist, const uint32_t* cand_packed,
                int32_t k, int32_t max_segment, int64_t max_iterations, int32_t threads, int32_t* status,
                int64_t* stats, void* stream);
int tspb_or_opt_max_n(void);

/* Coordinate-based TSPLIB edge weight types (src/distances/matrix.py:39-41). */
#define TSPB_EDGE_EUC_2D 0
#define TSPB_EDGE_EUC_3D 1
#define TSPB_EDGE_MAN_2D 2
#define TSPB_EDGE_MAN_3D 3
#define TSPB_EDGE_MAX_2D 4
#define TSPB_EDGE_MAX_3D 5
#define TSPB_EDGE_CEIL_2D 6
#define TSPB_EDGE_ATT 7
#define TSPB_EDGE_GEO 8
#define TSPB_EDGE_XRAY1 9

/*
 * Dense n x n int32 distance matrix (row stride ld) of one TSPLIB edge type from n x dim
 * float64 coordinates (dim 2 or 3; XRAY1 needs 3; the planar and 3-D formulas run over
 * all dim columns, GEO reads DDD.MM latitude and longitude from columns 0 and 1), zero
 * diagonal. Replaces compute_distance_matrix (src/distances/matrix.py:44-131, 214-273)
 * and the device formulas of pairwise_device.cuh; bit-identical for every type but GEO,
 * whose cos/acos may differ from the host's in the last bit (an entry changes only when
 * its value lies within about 1e-11 of an integer before truncation).
 */
int tspb_distance_matrix(const double* coords, int32_t n, int32_t dim, int32_t edge_type, int32_t* out, int64_t ld,
                         void* stream);

/*
 * Uniform random-permutation initial population, CTA per row: row r is `customers`
 * (n entries; NULL means 0..n-1) shuffled by Fisher-Yates from position n-1 down to 1,
 * position i swapped with the SplitMix64 bounded draw in [0, i] of the stream seeded with
 * seeds[r]. Replaces InitializationCPUPermRandom.initialize
 *   (src/algorithms/strategies/initialization/random_init.py:30-55) and random_init_kernel
 *   (.../initialization/kernels/random_init.cu).
 */
int tspb_random_init(const uint64_t* seeds, int32_t rows, int32_t n, const int32_t* customers, int32_t* out,
                     void* stream);
/* The same for many instances in one launch (customers 0..n-1 of each job; the jobs'
 * `k` and `cand` are ignored); max_n and max_rows bound every job's n and rows. */
int tspb_random_init_jobs(const tspb_nn_job* jobs, int32_t num_jobs, int32_t max_rows, int32_t max_n,
                          void* stream);

/*
 * The GA's random tape drawn exactly as NumPy's Generator(PCG64) draws it from
 * `context.rng` (src/utils/rng.py:48-64), in the reference's per-generation order:
 * tournament integers(0, P, (P, kt)) (tournament_selection.py:113), PMX cut pairs
 * sample_distinct_pairs(P/2, 0, n) (pmx_crossover.py:155), inversion random(P)
 * (inversion_mutation.py:82), inversion pairs sample_distinct_pairs(P, 0, n)
 * (route_helpers.py:214). `tspb_pcg64` holds bit_generator.state: the 128-bit state and
 * increment as (hi, lo) halves, has_uint32 and uinteger. The generator is advanced in
 * place; `states` (optional, [G]) receives the state after each generation.
 * tspb_tape_draw_host: one run on the host (plain C, no device).
 * tspb_tape_draw: `num` runs on the device, one thread per run; gens, ns, the tape
 *   arrays ([num][G][...]) and states ([num][G]) are device pointers.
 */
typedef struct tspb_pcg64 {
  uint64_t state_hi, state_lo, inc_hi, inc_lo;
  int32_t has_uint32;
  uint32_t uinteger;
} tspb_pcg64;
int tspb_tape_draw_host(tspb_pcg64* gen, int32_t G, int32_t P, int32_t kt, int32_t n, int32_t* tourn,
                        int32_t* cut_a, int32_t* cut_b, double* u, int32_t* inv_a, int32_t* inv_b,
                        tspb_pcg64* states);
int tspb_tape_draw(tspb_pcg64* gens, const int32_t* ns, int32_t num, int32_t G, int32_t P, int32_t kt,
                   int32_t* tourn, int32_t* cut_a, int32_t* cut_b, double* u, int32_t* inv_a, int32_t* inv_b,
                   tspb_pcg64* states, void* stream);

/*
 * One GA generation as graph-capturable steps. The random draws of all generations are
 * pre-drawn on the host in the reference's order and passed as a tape; `gen` (device
 * int) selects generation g's slice and is advanced by tspb_generation_track, `stopped`
 * (device int, set by the tracker when patience runs out) turns later steps into no-ops.
 *
 * tspb_generation_offspring: fused tournament selection, PMX crossover of pairs
 *   (2q, 2q+1), inversion mutation and closed-tour length of every child (CTA per child).
 *   Tape layout per generation: tourn [P][kt], cut_a/cut_b [P/2], u/inv_a/inv_b [P].
 *   Replaces SelectionCPUTournament.select_batch (tournament_selection.py:98-128),
 *   CrossoverCPUPermPartiallyMapped.crossover_batch (pmx_crossover.py:128-171),
 *   MutationCPUPermInversion.mutate_batch (inversion_mutation.py:65-99) and the offspring
 *   EvaluationStep (genetic_algorithm.py:174-199) of one generation.
 * tspb_generation_survival: stable (fitness, index) survival of [pop; off] into new_pop /
 *   new_fit; when the elite-th and (elite+1)-th survivors tie it sets tie_flags[g] = 1
 *   and *stopped = 2 (pause: the host decides the elite membership, then clears it).
 *   Replaces SurvivalStep / _select_survivors_assessed (genetic_algorithm.py:216-251, 618-706).
 * tspb_generation_elite_cost: fitness of rows [0, k) after the elite 2-opt
 *   (EliteOnlyLocalSearchStep re-evaluation, pipeline_steps.py:172-184).
 * tspb_generation_track: best-so-far with the strict 1e-6 rule, history[g+1], patience
 *   (genetic_algorithm.py:876-910).
 */
int tspb_generation_offspring(const int32_t* pop, const double* fit, int32_t P, int32_t n, int32_t kt,
                              const int32_t* tape_tourn, const int32_t* tape_cut_a, const int32_t* tape_cut_b,
                              const double* tape_u, const int32_t* tape_inv_a, const int32_t* tape_inv_b,
                              double rate, const int32_t* dist, int64_t dist_stride, const double* coords,
                              const int32_t* gen, const int32_t* stopped, int32_t* off, double* off_fit,
                              void* stream);
int tspb_generation_survival(const int32_t* pop, const double* fit, const int32_t* off, const double* off_fit,
                             int32_t P, int32_t n, int32_t elite, const int32_t* gen, int32_t* stopped,
                             int32_t* order, int32_t* new_pop, double* new_fit, int32_t* tie_flags, void* stream);
int tspb_generation_elite_cost(const int32_t* pop, int32_t k, int32_t n, const int32_t* dist, int64_t dist_stride,
                               const double* coords, const int32_t* stopped, double* fit, void* stream);
int tspb_generation_track(const double* fit, const int32_t* pop, int32_t P, int32_t n, int32_t* gen,
                          int32_t* stopped, int32_t* stall, int64_t patience, double* best_cost,
                          int32_t* best_tour, double* history, int32_t* done_gens, void* stream);

/*
 * Uneven multi-instance batch: many independent GA runs (one per instance, instances of
 * different sizes) advanced together, every generation of every run replayed from one
 * captured CUDA graph. No reference counterpart as a batch: each run computes exactly what
 * the tspb_generation_* steps compute for it alone (same tape layout, same survival, elite
 * and tracking rules); the runs progress independently through a per-instance control
 * block ctl[i] = {generation, state, stall, done}.
 *
 * States: RUN (the next launch sequence runs a whole generation), STOPPED (patience ran
 * out), PAUSED (the elite set is for the host to decide: it writes the elite rows to
 * host_elites[i] and sets RESUME), RESUME (the next launch sequence finishes the paused
 * generation with those elites, then continues), DONE (G generations ran).
 *
 * Elite-edge ties: when the elite-th and (elite+1)-th survivors tie, NumPy's unstable
 * argsort decides which tied rows are elites (EliteOnlyLocalSearchStep,
 * pipeline_steps.py:163). With the optional `clean` bits (1 = the row is a converged 2-opt
 * local optimum, whose refinement is skipped because it changes nothing), a tie whose rows
 * are all converged gives the same population for every choice and the run continues;
 * any other tie pauses the run.
 *
 * Phases of the 2-opt, cost and tracking steps: POSTINIT (every row of parity 0, no gate;
 * the post-init refinement), RESUME (runs in state RESUME, rows host_elites[i]), RUN (runs
 * in state RUN, rows [0, elite)), OFFSPRING (runs in state RUN, every offspring row of
 * `off`: the 2-opt of LocalSearchStep(target="offspring") that the reference's
 * local_search_stage="post_mutation" places between mutation and evaluation,
 * genetic_algorithm.py:254-277, 333-343; with `clean`, a converged child is skipped and
 * off_clean records the refinement's convergence).
 */
#define TSPB_BATCH_RUN 0
#define TSPB_BATCH_STOPPED 1
#define TSPB_BATCH_PAUSED 2
#define TSPB_BATCH_RESUME 3
#define TSPB_BATCH_DONE 4
#define TSPB_BATCH_HIT_OPTIMAL 5  /* best <= optimal + 1e-6 (stopped early) */
#define TSPB_BATCH_NEAR_OPTIMAL 6 /* (best - optimal) / optimal * 100 < 1 (stopped early) */

#define TSPB_BATCH_PHASE_POSTINIT 0
#define TSPB_BATCH_PHASE_RESUME 1
#define TSPB_BATCH_PHASE_RUN 2
#define TSPB_BATCH_PHASE_OFFSPRING 3

typedef struct tspb_batch_instance {
  int32_t n;                    /* cities, >= 4 */
  int32_t k;                    /* k-NN entries per row, 1 <= k <= n - 1 */
  int64_t pop_offset;           /* element offset of the P x n rows in pop[], off */
  int64_t node_offset;          /* element offset of the n-slot in best_tour */
  const int32_t* dist;          /* n x dist_stride int32, or NULL: distances from coords */
  int64_t dist_stride;
  const double* coords;         /* n x 2 float64; required when dist is NULL */
  const uint32_t* cand_packed;  /* n x k words c | d(a, c) << 16 (tspb_candidate_pack) */
  int64_t patience;             /* generations without a strict improvement before STOPPED */
  double optimal;               /* known optimal cost (> 0) for the early stops of
                                   genetic_algorithm.py:894-905, else 0 */
  const int32_t* rev_off;       /* reverse k-NN index (tspb_candidate_reverse_index), or NULL; */
  const int32_t* rev_idx;       /* required by TSPB_BATCH_INCREMENTAL */
} tspb_batch_instance;

typedef struct tspb_batch {
  int32_t num_instances;
  int32_t P;                /* population per instance, >= 2 */
  int32_t kt;               /* tournament size */
  int32_t elite;            /* elite rows refined per generation, 0..P */
  int32_t G;                /* generations on the tape */
  int32_t rows_max;         /* row slots per instance in ls_status / ls_stats (>= P) */
  double mutation_rate;
  const tspb_batch_instance* inst; /* device array [num_instances] */
  int32_t* pop[2];          /* populations; instance i at generation g reads pop[g & 1] */
  double* fit[2];           /* [I][P] */
  int32_t* off;             /* offspring rows (pop layout) */
  double* off_fit;          /* [I][P] */
  int32_t* order;           /* [I][P] survival scratch */
  const int32_t* tape_tourn; /* [I][G][P][kt] */
  const int32_t* tape_cut_a; /* [I][G][P/2] */
  const int32_t* tape_cut_b; /* [I][G][P/2] */
  const double* tape_u;      /* [I][G][P] */
  const int32_t* tape_inv_a; /* [I][G][P] */
  const int32_t* tape_inv_b; /* [I][G][P] */
  int32_t* ctl;             /* [I][4] generation, state, stall, done */
  double* best_cost;        /* [I] */
  int32_t* best_tour;       /* node_offset-indexed */
  double* history;          /* [I][G + 1] */
  int32_t* ties;            /* [I][G] elite-edge tie seen at generation g */
  const int32_t* host_elites; /* [I][elite] */
  int32_t* ls_status;       /* [I][rows_max] sticky 2-opt error of each row slot (0: none) */
  int64_t* ls_stats;        /* optional [I][rows_max][4] passes, pairs, moves, evaluated gains (accumulated) */
  uint8_t* clean[2];        /* optional [I][P] per population: 1 = converged 2-opt local optimum */
  uint8_t* off_clean;       /* [I][P] the same for the offspring (required with clean) */
  int32_t crossover;        /* TSPB_XOVER_PMX or TSPB_XOVER_OX */
  int32_t mutation;         /* TSPB_MUT_INVERSION or TSPB_MUT_SWAP */
} tspb_batch;

/* Fitness of every row of pop[parity]; with set_best also the initial best (first
 * minimum), history[i][0] and ctl (generation 0, RUN, or DONE when G == 0). */
int tspb_batch_init(const tspb_batch* b, int32_t parity, int32_t set_best, void* stream);
/* Offspring of generation ctl[i][0] for every RUN instance i in items[0..num_items), CTA
 * per child row, `threads` per CTA (32..256, multiple of 32); max_n bounds the items' n
 * (shared memory). Replaces SelectionCPUTournament.select_batch, CrossoverCPUPermPartiallyMapped
 * and MutationCPUPermInversion for every run (as tspb_generation_offspring). */
int tspb_batch_offspring(const tspb_batch* b, const int32_t* items, int32_t num_items, int32_t max_n,
                         int32_t threads, void* stream);
/* Survival of every RUN instance and the elite-edge tie rule (RUN -> PAUSED); replaces
 * _select_survivors_assessed (genetic_algorithm.py:618-706) for every run. */
int tspb_batch_survival(const tspb_batch* b, void* stream);
#define TSPB_BATCH_COORDS 1  /* every item has dist == NULL: distances rebuilt from coordinates */
#define TSPB_BATCH_GROUPED 2 /* every item's k is a multiple of 4 and its packed table 16-byte aligned */
/* with GROUPED: every item has rev_off/rev_idx. Best mode keeps the minimum improving key
 * of every row and, after a move with window [bi, bj], recomputes only the rows of the
 * window and the earlier rows with a candidate in it (30 n bytes of shared memory per
 * CTA instead of 16 n); first mode restarts from the move's row after checking the
 * affected entries (as tspb_two_opt with the reverse index). Same results either way. */
#define TSPB_BATCH_INCREMENTAL 4
/* best mode, GROUPED, not INCREMENTAL: every row is refined by a two-CTA thread-block
 * cluster; both CTAs keep the tour state and apply every move, each scans alternate
 * rounds of a pass, and the pass minimum is exchanged through distributed shared memory.
 * Same results; for phases with fewer units than SMs (elites of a few runs). threads counts
 * per CTA, and tspb_batch_two_opt_occupancy then reports co-resident CTAs of such pairs. */
#define TSPB_BATCH_PAIR 8
/* 2-opt over the (item, row) units of one phase: persistent CTAs (ctas <= 0: every CTA
 * that fits) take units from the device counter `queue` (zeroed by this call) in item
 * order; put the largest instances first. `flags` (TSPB_BATCH_*) state what holds for
 * every item; an item that disagrees gets TSPB_ERR_UNSUPPORTED in ls_status and is left
 * unchanged. mode BEST or FIRST, candidate mode only, threads 64/128/256/512/1024. In the
 * RESUME, RUN and OFFSPRING phases every refined row's fitness (fit or off_fit) is
 * rewritten from the final tour, the exact int64 sum of its edges; converged rows that are
 * skipped keep theirs.
 * Replaces the post-init and elite refinement calls of LocalSearchCPUTourTwoOpt
 * (pipeline_steps.py:103-125, 153-195) for every run. */
int tspb_batch_two_opt(const tspb_batch* b, const int32_t* items, int32_t num_items, int32_t max_n,
                       int32_t flags, int32_t phase, int32_t mode, int64_t max_iterations, int32_t threads,
                       int32_t ctas, uint32_t* queue, void* stream);
/* Resident CTAs per SM of tspb_batch_two_opt for this shape and flags (0: does not fit). */
int tspb_batch_two_opt_occupancy(int32_t max_n, int32_t mode, int32_t threads, int32_t flags);
/* Best tracking, history, early stops and the generation counter of a phase's instances:
 * RUN/RESUME -> HIT_OPTIMAL, NEAR_OPTIMAL, STOPPED (patience), DONE or RUN, checked in
 * that order (genetic_algorithm.py:876-910). */
int tspb_batch_track(const tspb_batch* b, int32_t phase, void* stream);

/*
 * k-nearest-neighbour table on the device (CTA per node): out[u][0..k) ordered by
 * (distance, node id), self excluded, k <= 64. Counterpart of compute_candidate_list
 *   (src/distances/matrix.py:140-211) with a fixed tie rule (lower id wins at the k-th
 *   boundary) where the reference's argpartition leaves the winner unspecified; used for
 *   bulk preprocessing, while the 2-opt strategies keep the context's host table.
 */
int tspb_knn(const int32_t* dist, int64_t dist_stride, const double* coords, int32_t n, int32_t k,
             int32_t* out, void* stream);
/* The same table (k + 1 <= 64) and ties[u] = 1 where the k-th and (k+1)-th nearest
 * distances of u are equal: only those rows can differ from the reference's argpartition,
 * every other row equals compute_candidate_list's. */
int tspb_knn_ties(const int32_t* dist, int64_t dist_stride, const double* coords, int32_t n, int32_t k,
                  int32_t* out, int32_t* ties, void* stream);

/*
 * Learned candidate lists (no reference counterpart: the reference uses plain k-NN).
 * Edge-scoring MLP 5 -> 64 -> 64 -> 1, FP32 master parameters used in BF16, FP32
 * accumulation, tensor-core layers (mma.sync bf16). Parameter block of
 * tspb_mlp_param_count() floats: W1[16][64] (rows >= 5 zero), b1[64], W2[64][64], b2[64],
 * w3[64], b3.
 * tspb_edge_features: x (n*pool_k rows of 16 bf16) for candidate edges (u, pool[u][s]):
 *   d/s_u, s/pool_k, rank of u in pool[v] / pool_k, dx/s_u, dy/s_u, s_u = d(u, pool[u][-1]);
 *   labels (optional) = 1 when v is next to u in the tour given by tour_pos (node -> position).
 * tspb_mlp_infer: logits of num_edges rows.
 * tspb_mlp_train_grad: adds d(mean BCE-with-logits)/dparams over the batch to grad and
 *   the summed loss to *loss.
 * tspb_mlp_adam: one Adam step on params from grad (grad is zeroed).
 * tspb_select_topk: out[u][0..k) = pool entries of u with the highest scores.
 */
int tspb_mlp_param_count(void);
int tspb_edge_features(const double* coords, int32_t n, const int32_t* pool, int32_t pool_k,
                       const int32_t* dist, int64_t dist_stride, const int32_t* tour_pos, uint16_t* x,
                       float* labels, void* stream);
int tspb_mlp_infer(const float* params, const uint16_t* x, int64_t num_edges, float* logits, void* stream);
int tspb_mlp_train_grad(const float* params, const uint16_t* x, const float* labels, int64_t num_edges,
                        float* grad, float* loss, void* stream);
/*
 * tspb_mlp_train_grad on the fifth-generation tensor cores (tcgen05, accumulators in tensor
 * memory): the same gradient, with the hidden-layer products, the back-propagation
 * product and the weight-gradient sums over the batch as tcgen05 MMAs on 128-edge tiles.
 * One more rounding point than tspb_mlp_train_grad: dh1 enters dW1 and db1 in BF16. x must
 * be 16-byte aligned. status (optional) receives TSPB_ERR_BUDGET if an MMA completion wait
 * runs out (about a second). No reference counterpart (the reference has no learned lists).
 */
int tspb_mlp_train_grad_tc(const float* params, const uint16_t* x, const float* labels, int64_t num_edges,
                           float* grad, float* loss, int32_t* status, void* stream);
int tspb_mlp_adam(float* params, float* grad, float* m, float* v, int32_t step, float lr, float beta1,
                  float beta2, float eps, float weight_decay, void* stream);
int tspb_select_topk(const int32_t* pool, const float* scores, int32_t n, int32_t pool_k, int32_t k,
                     int32_t* out, void* stream);

/*
 * Permutation check: bad[r] = 0 when row r is a permutation of 0..n-1, else 1.
 */
int tspb_validate_perm(const int32_t* tours, int32_t num_tours, int32_t n, int32_t* bad, void* stream);

/*
 * Dense EUC_2D matrix from FP64 coordinates: nint(sqrt(dx*dx + dy*dy)) with separate
 * IEEE multiplies and add (no FMA), zero diagonal. Replaces compute_distance_matrix
 *   (src/distances/matrix.py:84-86, 214-273) and gpu_euc_2d
 *   (src/distances/kernels/pairwise_device.cuh:58-60).
 */
int tspb_euc2d_matrix(const double* coords, int32_t n, int32_t* dist, int64_t dist_stride, void* stream);

/*
 * Roofline microbenchmarks (no counterpart in the reference; they measure the ceilings of
 * the L2-resident 2-opt scan on the machine at hand). Time each launch with CUDA events.
 *   tspb_microbench_l2_gather: blocks x 256 threads x iters x 8 random 4-byte loads
 *     (L1 bypassed, one 32-byte L2 sector each) from table[0, table_len), table_len a
 *     power of two; size the table to fit L2 (the scan's 4 MB matrix does).
 *   tspb_microbench_int32: blocks x 256 threads x iters x 128 integer instructions
 *     (alternating add.s32 / xor.b32 over eight independent chains per thread).
 * `sink` receives at most one store; it only keeps the work from being optimised away.
 */
int tspb_microbench_l2_gather(const int32_t* table, int64_t table_len, int32_t iters, int32_t blocks, int32_t* sink,
                              void* stream);
int tspb_microbench_int32(int32_t iters, int32_t blocks, int32_t seed, int32_t* sink, void* stream);

/*
 * CUDA graphs of this library's launches (no counterpart in the reference, whose GA loop
 * launches every kernel from Python each generation: genetic_algorithm.py:789-965).
 *   tspb_graph_capture_begin: start capturing `stream` (not the legacy default stream),
 *     relaxed mode; every tspb_* launch on that stream until the end call is recorded.
 *   tspb_graph_capture_end: end the capture, instantiate and upload the graph; *exec_out
 *     receives the executable graph (TSPB_ERR_CUDA and NULL if the capture was invalidated).
 *   tspb_graph_launch: replay it on `stream`.
 *   tspb_graph_destroy: free it (a replay still running finishes first).
 * The captured launches keep the device pointers they were given: a replay reads and
 * writes the same buffers, which must outlive the executable graph.
 */
int tspb_graph_capture_begin(void* stream);
int tspb_graph_capture_end(void* stream, void** exec_out);
int tspb_graph_launch(void* exec, void* stream);
int tspb_graph_destroy(void* exec);

#ifdef __cplusplus
}
#endif

#endif /* TSPB_H */
