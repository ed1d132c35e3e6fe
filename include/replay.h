/* replay.h -- C ABI of libreplay, the B200 (sm_100a) engine for Monte Carlo
 * SEIR replay over temporal contact networks.
 *
 * The reference (HarrisonGreenlee/Replay) exposes no library API: its
 * boundary is the `replay` executable (tool/gpu_cpu_temporal_sim.cu:570-699)
 * plus an internal C ABI for ingest (tool/temporal_contact_matrix.h:58-94).
 * Every entry point below names the reference interface it replaces.  The
 * `replay` executable built beside this library keeps the reference's flags,
 * defaults and CSV outputs and is implemented on top of these calls.
 *
 * Conventions: plain pointers and sizes, no C++ or torch types; every call
 * returns an rp_status (no exit()); rp_last_error() describes the last
 * failure on the calling thread.  Handles are not thread-safe; distinct
 * handles may be used from distinct threads.  Device memory is owned by the
 * handle; host arrays are owned by the caller.  The one process-wide state
 * is a thread-safe cache of device blocks: freeing a graph, simulation or
 * mean-field handle synchronizes the device and keeps its blocks (up to
 * 8 GiB per device) for the next handle instead of returning them with
 * cudaFree; rp_release_cached_memory() returns them.
 */
#ifndef REPLAY_H
#define REPLAY_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define RP_API __attribute__((visibility("default")))
#else
#define RP_API
#endif

typedef enum {
  RP_OK = 0,
  RP_ERR_ARG = 1,    /* invalid argument or unsupported combination */
  RP_ERR_IO = 2,     /* file cannot be opened or read */
  RP_ERR_PARSE = 3,  /* malformed contact file (the reference exits 1) */
  RP_ERR_NOMEM = 4,  /* host or device allocation failed */
  RP_ERR_CUDA = 5,   /* CUDA runtime error */
  RP_ERR_RANGE = 6,  /* size or time arithmetic out of range */
  RP_ERR_DEVICE = 7  /* a kernel raised its error flag */
} rp_status;

/* Message for the last failed call on this thread ("" if none). */
RP_API const char *rp_last_error(void);
/* Library version string. */
RP_API const char *rp_version(void);
/* Returns every device block kept from freed handles to the driver
 * (cudaFree), on every device.  No reference counterpart. */
RP_API void rp_release_cached_memory(void);

/* ------------------------------------------------------------------------ */
/* Contact graphs.                                                           */
/* ------------------------------------------------------------------------ */
typedef struct rp_graph rp_graph;

typedef struct {
  int32_t n_nodes;     /* NODE_LIST token count: the simulated population N */
  int32_t n_index;     /* distinct contact endpoints seen in contact lines */
  int64_t n_contacts;  /* parsed contacts (intervals) */
  int64_t nlists;      /* the reference interval database's sublist count */
  int64_t n_malformed; /* skipped contact lines ("malformed line skipped") */
  int64_t t_min;       /* smallest stored start */
  int64_t t_max;       /* largest stored end */
  int32_t n_classes;   /* duration classes of the interval index */
  int32_t device;      /* CUDA device holding the index */
  double prep_ms;      /* host time: argument checks, endpoint pass (from arrays) or parse (text) */
  double build_ms;     /* host time of the upload and device index build (synchronised) */
} rp_graph_info;

/* Parses a contact file (NODE_LIST header, then `u, v, ISO8601, ISO8601;`
 * lines) and builds the device interval index.
 * Replaces parse_edgelist_build_intervals + build_interval_db_wrapper
 * (tool/temporal_contact_matrix.c:148-321, :377-392). */
RP_API rp_status rp_graph_load_text(const char *path, int device,
                                    rp_graph **out);

/* Builds a graph from arrays already in memory: contact k joins compressed
 * node indices u[k], v[k] (0 <= u,v < n_nodes) over [start[k], end[k]) in
 * integer seconds.  Replaces the IntervalMap array the reference builds in
 * tool/temporal_contact_matrix.c:262-313. */
RP_API rp_status rp_graph_from_arrays(const int64_t *start, const int64_t *end,
                                      const int32_t *u, const int32_t *v,
                                      int64_t n_contacts, int32_t n_nodes,
                                      int device, rp_graph **out);

/* Parses a contact file into host arrays only (no device is touched), with
 * the same rules as rp_graph_load_text: u[k] <= v[k] are compressed node
 * indices in order of first appearance, start/end in Unix seconds, file
 * order kept.  The four arrays are allocated by the library (NULL when
 * *n_contacts is 0) and released with rp_free.
 * Replaces parse_edgelist_build_intervals
 * (tool/temporal_contact_matrix.c:148-321). */
RP_API rp_status rp_parse_contacts(const char *path, int32_t *n_nodes,
                                   int32_t *n_index, int64_t *n_contacts,
                                   int64_t *n_malformed, int64_t **start,
                                   int64_t **end, int32_t **u, int32_t **v);
/* Releases an array returned by rp_parse_contacts. */
RP_API void rp_free(void *p);

RP_API rp_status rp_graph_get_info(const rp_graph *g, rp_graph_info *out);

/* Frees the graph.  Replaces free_interval_db_wrapper + free_node_map
 * (tool/temporal_contact_matrix.c:394-403, :364-372). */
RP_API void rp_graph_free(rp_graph *g);

/* Window CSR test hook: the symmetric CSR the step loop multiplies for the
 * window [ws, we), built on the device and copied back in canonical form
 * (rows ascending, columns ascending, duplicates merged).
 * weight_kind 0: FP32 weights (float)overlap * scale, merged by sequential
 *   FP32 adds in hit order -- build_csr_from_intervals
 *   (tool/gpu_cpu_temporal_sim.cu:238-350) fed by find_intervals
 *   (tool/gpu_cpu_temporal_sim.cu:973-991);
 * weight_kind 1: int32 contact-second weights (scale ignored).
 * ncls_cap 1 applies the reference driver's max(nlists,1) hit cap.
 * `val` is float* or int32_t* by weight_kind; col/val hold `capacity`
 * entries; row_ptr holds n_nodes+1.  *nnz and *n_hits are always set; the
 * call fails with RP_ERR_RANGE if nnz exceeds capacity. */
RP_API rp_status rp_window_csr(rp_graph *g, int64_t ws, int64_t we,
                               float scale, int32_t weight_kind,
                               int32_t ncls_cap, int32_t *row_ptr,
                               int32_t *col, void *val, int64_t capacity,
                               int64_t *nnz, int64_t *n_hits);

/* Allocation-free variant of rp_window_csr, with no counterpart in the
 * reference: builds the same window CSR on the device and leaves it in
 * caller-owned device buffers -- d_row_ptr (n_nodes+1 int32) and d_entries
 * (`capacity` pairs {col, weight} of int32, weight as rp_window_csr's
 * weight_kind) -- without allocating or freeing device memory.  For callers
 * that cannot pay cudaFree's device-wide wait per window or that hand all
 * device memory to their own pool.  Scratch is one static device array
 * (about 9 MB per device), so the graph may have at most 65,536 nodes and
 * the window at most 131,072 candidate contacts (RP_ERR_RANGE beyond).
 * Calls share that scratch: concurrent or overlapping calls race, so issue
 * them one at a time.  Each call looks the scratch up (cudaGetSymbolAddress),
 * copies small descriptors from the host and synchronizes `stream` before it
 * returns, so it must not be made while `stream` is being captured.  The
 * caller's current device is restored.  Returns when the CSR is in place;
 * *nnz and *n_hits as for rp_window_csr. */
RP_API rp_status rp_window_csr_noalloc(rp_graph *g, int64_t ws, int64_t we,
                                       float scale, int32_t weight_kind,
                                       int32_t ncls_cap, int32_t *d_row_ptr,
                                       int32_t *d_entries, int64_t capacity,
                                       int64_t *nnz, int64_t *n_hits,
                                       void *stream);

/* ------------------------------------------------------------------------ */
/* Simulations.                                                              */
/* ------------------------------------------------------------------------ */
typedef struct rp_sim rp_sim;

enum {
  RP_TRANSITION_COUNTDOWN = 0, /* the reference's deterministic countdowns */
  RP_TRANSITION_GEOMETRIC = 1  /* per-step Bernoulli E->I, I->R, R->S */
};
enum {
  RP_PATH_AUTO = 0,    /* batched for geometric, plain for countdown */
  RP_PATH_PLAIN = 1,   /* per-replica SpMV + elementwise transition */
  RP_PATH_BATCHED = 2  /* replica-bit-packed SpMM fused with transitions */
};
enum {
  RP_CSR_PER_STEP = 0, /* build each window's CSR inside the step loop */
  RP_CSR_PREBUILT = 1  /* build every window's CSR once, then replay */
};

typedef struct {
  uint32_t struct_size; /* sizeof(rp_params); set by rp_params_default */
  int32_t n_replicas;   /* --M (default 1000) */
  int32_t n_steps;      /* --iterations (default 42) */
  float step_size;      /* --step-size seconds (default 3600) */
  int64_t start_time;   /* --start-time (default 946713600) */
  int64_t window;       /* --static-network-duration (default 3600) */
  int32_t transition;   /* RP_TRANSITION_* (default countdown) */
  int32_t path;         /* RP_PATH_* (default auto) */
  int32_t csr_mode;     /* RP_CSR_* (default per step) */
  int32_t ncls_cap;     /* apply the reference's hit cap (default 1) */
  uint64_t seed;        /* counter-based random stream key (default 1) */
  /* countdown mode (reference semantics) */
  int32_t exposed_duration;    /* --exposed-duration */
  int32_t infectious_duration; /* --infectious-duration */
  int32_t resistant_duration;  /* --resistant-duration */
  float infect_prob;           /* --infect-prob: per exposure-hour */
  /* initial condition */
  float initial_infected; /* --initial-infected: Bernoulli probability */
  int32_t initial_count;  /* > 0: exactly this many per replica instead */
  /* geometric mode */
  float beta;                    /* per contact-second */
  const float *beta_per_replica; /* host, n_replicas values, or NULL */
  const float *susceptibility;   /* host, n_nodes values, or NULL */
  float p_ei;          /* E->I probability per step */
  float p_ir;          /* I->R probability per step */
  float p_rs;          /* R->S probability per step (0: no waning) */
  int32_t has_exposed; /* 0: S->I directly (SIR/SIS) */
  int32_t ir_to_s;     /* 1: recovery returns to S (SIS) */
  int32_t record_node_states; /* keep per-step node states for callbacks */
  int32_t replica_offset; /* replicas 0..M-1 draw the random streams of
                           * replicas replica_offset..+M-1 (a multiple of 32):
                           * disjoint shards of one replica range, run on any
                           * GPUs, reproduce the unsharded run exactly.  Not
                           * in the reference. */
} rp_params;

/* Fills the reference's defaults (tool/gpu_cpu_temporal_sim.cu:24-56). */
RP_API void rp_params_default(rp_params *p);

/* Allocates device state for one replay of `g` with `p`.  Replaces the
 * set-up in tool/gpu_cpu_temporal_sim.cu:753-857. */
RP_API rp_status rp_sim_create(const rp_graph *g, const rp_params *p,
                               rp_sim **out);
/* Independent networks of uneven size batched into one replay (no
 * reference counterpart; the reference runs one network per process).  The
 * graph holds the union of the networks, network k owning the nodes
 * [net_first[k], net_first[k+1]) (n_networks+1 offsets, from 0 to the
 * graph's n_nodes); contacts between networks would couple them.  All
 * networks share the schedule and every parameter; initial_count applies to
 * each (network, replica).  Counts are (n_steps+1) x n_networks x
 * n_replicas x 4.  Batched (geometric) path only, with ncls_cap = 0: the
 * reference's hit cap is a property of one network's own index. */
RP_API rp_status rp_sim_create_batch(const rp_graph *g, const rp_params *p,
                                     const int32_t *net_first,
                                     int32_t n_networks, rp_sim **out);
RP_API void rp_sim_free(rp_sim *s);

/* Per-step node states: states[r * n_nodes + i] in {0 susceptible,
 * 1 exposed/incubating, 2 infectious, 3 resistant}, replica-major as the
 * reference's node CSV rows.  step_index 0 is the initial state; a non-zero
 * return aborts the run. */
typedef int (*rp_state_cb)(void *user, int32_t step_index, int64_t timestamp,
                           const uint8_t *states, int32_t n_nodes,
                           int32_t n_replicas);

/* Runs the whole replay: initial state, then n_steps steps.  counts receives
 * (n_steps+1) x n_replicas x 4 int32 (exposed, infectious, resistant,
 * susceptible), row 0 the initial state.  `cb` may be NULL; it is called
 * only when record_node_states is set.  Replaces the step loop of
 * tool/gpu_cpu_temporal_sim.cu:859-1150. */
RP_API rp_status rp_sim_run(rp_sim *s, int32_t *counts, rp_state_cb cb,
                            void *user);

/* Node-state CSV text, formatted on the device: `cb` receives, for every
 * recorded step (step_index 0 the initial state), the lines
 * "time,simulation_id,node_id,state\n" (state susceptible, incubating,
 * infectious or resistant) with replicas outer and nodes inner, in one or
 * more chunks of whole lines (about 64 MB each); the device formats the
 * next chunk while the callback handles the current one.  Needs
 * record_node_states.  Replaces the node rows of write_simulation_state
 * (tool/gpu_cpu_temporal_sim.cu:505-568). */
typedef int (*rp_text_cb)(void *user, int32_t step_index, int64_t timestamp,
                          const char *text, size_t len);
RP_API rp_status rp_sim_run_text(rp_sim *s, int32_t *counts, rp_text_cb cb,
                                 void *user);

/* Device-resident replay on a CUDA stream (cudaStream_t, or NULL for the
 * legacy stream): re-initialises the state and enqueues every step; counts
 * stay on the device (rp_sim_counts copies them).  No host synchronisation. */
RP_API rp_status rp_sim_enqueue(rp_sim *s, void *stream);
RP_API rp_status rp_sim_counts(rp_sim *s, int32_t *counts);
/* Timestamps of the count rows: ts[0] = start_time, ts[k] = the start of
 * step k-1 (the reference writes row 1 at start_time as well). */
RP_API rp_status rp_sim_timestamps(rp_sim *s, int64_t *ts);

typedef struct {
  int32_t path;          /* resolved RP_PATH_* */
  int32_t words;         /* replica words per node (batched path) */
  int32_t n_windows;     /* distinct network windows */
  int32_t kernels_per_run; /* kernel launches one replay enqueues */
  int64_t max_candidates;  /* most index candidates of any window */
  int64_t prebuilt_nnz;    /* total CSR entries when prebuilt */
  int64_t device_bytes;    /* device memory the handle holds */
  int64_t nnz_total;       /* sum over steps of CSR entries multiplied */
  /* host time of rp_sim_create's phases, ms */
  double setup_ms;         /* schedule, window plans, window workspaces */
  double alloc_ms;         /* state, counters and count buffers */
  double prebuild_ms;      /* every window CSR built once (prebuilt mode) */
  double capture_ms;       /* CUDA graph capture and instantiation */
} rp_sim_info;
RP_API rp_status rp_sim_get_info(const rp_sim *s, rp_sim_info *out);

/* Per-kernel-group device time of one eager (not graph-launched) replay,
 * measured with CUDA events on the simulation's stream.  No reference
 * counterpart: the reference only prints wall-clock progress. */
typedef struct {
  double total_ms;         /* whole replay */
  double build_ms;         /* window CSR builds */
  double spmv_ms;          /* plain path: per-replica SpMV */
  double step_ms;          /* batched step kernel / plain transition kernel */
  double other_ms;         /* initial state, counts, finalize */
  int32_t step_launches;   /* launches counted in step_ms */
  int32_t spmv_launches;
  int32_t build_launches;  /* window builds (each several kernels) */
  int32_t kernels;         /* all kernel launches of the replay */
} rp_profile;
RP_API rp_status rp_sim_profile(rp_sim *s, rp_profile *out);
/* Device time of each step's exposure + transition kernels (n_steps floats,
 * ms) from the same eager replay; no reference counterpart. */
RP_API rp_status rp_sim_profile_steps(rp_sim *s, float *step_ms);

/* Tile autotuner of the batched path (no reference counterpart).  Networks
 * are bucketed by size (floor(log2 nodes)); for each bucket, largest first,
 * the task height (rows of one task: 32..4096) and then the staging depth
 * (CSR pairs the exposure kernel stages per chunk: 192, 384 or the default
 * 768) are chosen by timing the replay's first `probe_steps` steps with
 * CUDA events, keeping a candidate only when it is 2% faster.  The
 * simulation keeps the tuned tiles (and re-captures its CUDA graph); results
 * are unchanged by tiling.  Not for simulations created with
 * record_node_states. */
typedef struct {
  int32_t n_buckets;         /* network-size buckets */
  int32_t bucket_log2[32];   /* floor(log2 nodes) of each bucket */
  int32_t rows_per_task[32]; /* chosen task height, 0 = default kept */
  int32_t stage_pairs[32];   /* chosen staging depth, 0 = default kept */
  int32_t probe_steps;       /* steps per timed probe */
  int32_t probes;            /* configurations timed */
  double ms_default;         /* probe time with the default tiles */
  double ms_tuned;           /* probe time with the chosen tiles */
} rp_tune_result;
RP_API rp_status rp_sim_autotune(rp_sim *s, int32_t probe_steps,
                                 rp_tune_result *out);

/* ------------------------------------------------------------------------ */
/* Expected-value (mean-field) replay and its adjoint.  No reference        */
/* counterpart: the differentiable form of the geometric replay.            */
/* ------------------------------------------------------------------------ */
typedef struct rp_meanfield rp_meanfield;

/* Builds the schedule and every window CSR (int32 contact-second weights) of
 * the replay described by p: n_steps, step_size, start_time, window,
 * ncls_cap, has_exposed and ir_to_s are used; replica and rate fields are
 * ignored.  The adjoint recomputes states between checkpoints taken every
 * `checkpoint_every` steps.  The graph must outlive the handle. */
RP_API rp_status rp_meanfield_create(const rp_graph *g, const rp_params *p,
                                     int32_t checkpoint_every,
                                     rp_meanfield **out);
RP_API void rp_meanfield_free(rp_meanfield *m);

/* Forward replay on device pointers, enqueued on `stream`.  x0: 4*N floats,
 * the planes S, E, I, R of node probabilities.  Per step, with
 * e_i = scale * sum_j w_ij I_j and P_i = 1 - exp(-beta s_i e_i):
 * S' = S(1-P) + p_rs R, E' = E(1-p_ei) + S P, I' = I(1-p_ir) + p_ei E,
 * R' = R(1-p_rs) + p_ir I (S->I directly without an exposed state; I->S
 * with ir_to_s).  d_susceptibility: N floats, or NULL for all ones.
 * d_incidence (n_steps floats): expected new infections sum_i S_i P_i of
 * each step; d_xT (4*N floats, optional): the final planes.  Keeps the
 * checkpoints and parameters for rp_meanfield_backward. */
RP_API rp_status rp_meanfield_forward(rp_meanfield *m, const float *d_x0,
                                      float beta, const float *d_susceptibility,
                                      float p_ei, float p_ir, float p_rs,
                                      float *d_incidence, float *d_xT,
                                      void *stream);

/* Reverse-time adjoint of the last forward: given dL/dincidence (n_steps
 * floats, or NULL for zeros) and dL/dx_T (4*N, or NULL), writes dL/dx0
 * (4*N floats), dL/dsusceptibility (N floats, optional) and d_grad_rates =
 * dL/d(beta, p_ei, p_ir, p_rs) as 4 doubles on the device (optional; the
 * scalar reductions run in FP64).  Transpose products use the same CSRs
 * (window graphs are symmetric). */
RP_API rp_status rp_meanfield_backward(rp_meanfield *m,
                                       const float *d_grad_incidence,
                                       const float *d_grad_xT, float *d_grad_x0,
                                       float *d_grad_susceptibility,
                                       double *d_grad_rates, void *stream);

/* ------------------------------------------------------------------------ */
/* Kernel test hooks on device pointers.                                     */
/* ------------------------------------------------------------------------ */

/* Plain per-replica SpMV, the drop-in for the reference's cusparseSpMM
 * (tool/gpu_cpu_temporal_sim.cu:1062-1064): exposure[i + r*n] =
 * sum_k val[k] * infectious[col[k] + r*n], sequential FP32 row sums in CSR
 * order (the order Eigen's CPUComputeSpMM uses, :403-433). */
RP_API rp_status rp_exposure_spmv_f32(const int32_t *d_row_ptr,
                                      const int32_t *d_col,
                                      const float *d_val, int32_t n_nodes,
                                      const float *d_infectious,
                                      float *d_exposure, int32_t n_replicas,
                                      void *stream);

/* Replica-bit-packed SpMM: masks[j * words + w] bit b marks replica
 * 32*w + b of node j infectious; exposure[i * n_replicas + r] receives the
 * exact int64 contact-second sum.  Entries are CSR pairs {col, weight}. */
RP_API rp_status rp_exposure_spmm_packed(const int32_t *d_row_ptr,
                                         const int32_t *d_entries,
                                         int32_t n_nodes,
                                         const uint32_t *d_masks,
                                         int32_t words, int32_t n_replicas,
                                         int64_t *d_exposure, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* REPLAY_H */
