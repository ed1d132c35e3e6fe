/* CPU oracle for the replay hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's algorithm (HarrisonGreenlee/Replay,
 * tool/temporal_contact_matrix.c, tool/ncls/ncls/src/intervaldb.c and
 * tool/gpu_cpu_temporal_sim.cu), plus the counter-based random streams and
 * the geometric transition mode that the CUDA path adds.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as the
 * checker; the product never links or calls it.
 *
 * Parity pinning: the parser, the NCLS window query (including its hit cap),
 * the CSR builder, the SpMM and the countdown rules are checked against the
 * reference built from its own sources (oracle/_ref) and against golden
 * fixtures generated from it (tests/golden/).
 */
#ifndef REPLAY_ORACLE_H
#define REPLAY_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- counter-based random numbers ---------------------------------------- *
 * key = seed; counter = (node, step, c2, c3):
 *   countdown infection uniform of replica r: c2 = r / 4, c3 = 3, output
 *     r % 4, as the 24-bit grid value ((x >> 8) + 1) 2^-24; event iff P > u;
 *   geometric infection uniform of replica r: top 8 bits bit-sliced on
 *     c2 = r / 32, c3 = 4 | j << 4, low 56 bits on c2 = r, c3 = 12
 *     (orc_infect_event); event iff U < floor(P 2^64);
 *   flow (E->I, I->R, R->S) uniform of replica r: bit-sliced, see
 *     orc_flow_event;
 *   initial Bernoulli: step = 0xFFFFFFFF, c2 = r / 4, c3 = 1;
 *   initial exact count (Floyd): node = draw j, step = 0xFFFFFFFE, c2 = r,
 *     c3 = 2. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2],
                       uint32_t out[4]);
float orc_unit(uint32_t x); /* ((x>>8)+1) * 2^-24, in (0,1] */
float orc_uniform(uint64_t seed, uint32_t node, uint32_t step,
                  uint32_t replica, uint32_t stream);
float orc_one_minus_exp_neg(float x);
uint64_t orc_threshold64(float p, int *always);
int orc_infect_event(uint64_t seed, uint32_t node, uint32_t step, uint32_t replica, float P);
int orc_flow_event(uint64_t seed, uint32_t node, uint32_t step, uint32_t replica,
                   uint64_t T, int always);

/* ---- ingest ---------------------------------------------------------------- */
int64_t orc_timegm(int year, int month0, int mday, int hour, int min, int sec);
int64_t orc_parse_iso8601(const char *s);
/* Parses a contact file.  Returns 0 on success, else a positive error code
 * (1 open, 2 header, 3 node list, 4 no edges, 5 more parsed than counted).
 * Arrays are malloc'd (free with orc_free). u/v are the (min,max) compressed
 * indices; n_index is the number of distinct contact endpoints seen. */
int orc_parse_file(const char *path, int32_t *n_nodes, int32_t *n_index,
                   int64_t *n_contacts, int64_t **start, int64_t **end,
                   int32_t **u, int32_t **v, int64_t *n_malformed);
void orc_free(void *p);

/* ---- interval index --------------------------------------------------------- */
/* Stored coordinates of the reference's interval database: intervals with
 * start < 0 are mirrored to (-end, -(int32)start). */
void orc_store_coords(const int64_t *start, const int64_t *end, int64_t n,
                      int64_t *out_s, int64_t *out_e);
/* Coordinates a stored hit is handed to the CSR builder with, for a window
 * starting at ws (mirrored back when orientations differ). */
void orc_hit_coords(int64_t s, int64_t e, int64_t ws, int64_t *hs, int64_t *he);
/* Stable sort permutation by (start asc, end desc). */
void orc_sort_order(const int64_t *start, const int64_t *end, int64_t n,
                    int64_t *perm);
/* nlists of the reference's nested containment list over these contacts. */
int64_t orc_nlists(const int64_t *start, const int64_t *end, int64_t n);
/* Window query with the reference main loop's hit cap (max(nlists,1)).  Contacts must be
 * given in stored coordinates and sorted order (orc_sort_order).  Writes sorted positions of hits in
 * query order into out_rank (capacity n).  Returns the hit count. */
int64_t orc_window_hits(const int64_t *s_start, const int64_t *s_end, int64_t n,
                        int64_t nlists, int64_t ws, int64_t we,
                        int64_t *out_rank);

/* ---- window CSR ---------------------------------------------------------- */
/* Reference semantics (FP32 weights = (float)overlap * scale, duplicates
 * merged by sequential FP32 adds in hit order).  row_ptr: n_nodes+1; col/val:
 * capacity 2*n_hits.  Returns nnz. */
int64_t orc_csr_f32(const int64_t *s_start, const int64_t *s_end,
                    const int32_t *s_u, const int32_t *s_v,
                    const int64_t *hit_rank, int64_t n_hits, int32_t n_nodes,
                    int64_t ws, int64_t we, float scale, int32_t *row_ptr,
                    int32_t *col, float *val);
/* Integer contact-second weights (scale not applied), duplicates summed. */
int64_t orc_csr_i32(const int64_t *s_start, const int64_t *s_end,
                    const int32_t *s_u, const int32_t *s_v,
                    const int64_t *hit_rank, int64_t n_hits, int32_t n_nodes,
                    int64_t ws, int64_t we, int32_t *row_ptr, int32_t *col,
                    int32_t *val);

/* ---- exposure --------------------------------------------------------------- */
/* C[:,r] = A * B[:,r], column-major N x M, sequential row sums in CSR order. */
void orc_spmm_f32(const int32_t *row_ptr, const int32_t *col, const float *val,
                  int32_t n, const float *b, float *c, int32_t m);
void orc_spmm_i64(const int32_t *row_ptr, const int32_t *col,
                  const int32_t *val, int32_t n, const uint8_t *b, int64_t *c,
                  int32_t m);

/* ---- step schedule ------------------------------------------------------- */
/* Per-step window start/end, weight scale and timestamp, as the reference's
 * driver loop computes them.  Returns 0, or 1 on overflow / bad arguments. */
int orc_schedule(int64_t start_time, float step_size, int64_t window,
                 int32_t n_steps, int64_t *ws, int64_t *we, float *scale,
                 int64_t *ts);

/* ---- simulation ------------------------------------------------------------ */
typedef struct {
  int32_t n_replicas;
  int32_t n_steps;
  float step_size;
  int64_t start_time;
  int64_t window;
  int32_t transition; /* 0 countdown (reference), 1 geometric */
  uint64_t seed;
  /* countdown */
  int32_t exposed_duration, infectious_duration, resistant_duration;
  float infect_prob;
  /* initial condition */
  float initial_infected; /* Bernoulli probability */
  int32_t initial_count;  /* exact count per replica when > 0 */
  /* geometric */
  float beta;               /* per contact-second */
  const float *beta_per_replica; /* optional, length n_replicas */
  const float *susceptibility;   /* optional, length n_nodes */
  float p_ei, p_ir, p_rs;
  int32_t has_exposed; /* 0: S->I directly */
  int32_t ir_to_s;     /* 1: I->S (SIS) */
  int32_t ncls_cap;    /* 1: apply the reference's hit cap */
  /* optional batch of independent networks: network k owns the nodes
   * [net_first[k], net_first[k+1]); counts become per (network, replica) */
  const int32_t *net_first; /* n_nets + 1 offsets, or NULL for one network */
  int32_t n_nets;
  /* replica r of this run draws the streams of replica r + replica_offset
   * (a multiple of 32): shards of one replica range reproduce it exactly */
  int32_t replica_offset;
} orc_params;

/* Runs the whole replay.  counts: (n_steps+1) x n_nets x n_replicas x 4
 * int32 rows (n_nets = 1 without a batch) of
 * (exposed, infectious, resistant, susceptible); row 0 is the initial state.
 * Optional node_states: (n_steps+1) x n_replicas x n_nodes uint8 of
 * 0 susceptible, 1 exposed/incubating, 2 infectious, 3 resistant.
 * Contacts are given in file order.  Returns 0 or an error code. */
int orc_run(const int64_t *start, const int64_t *end, const int32_t *u,
            const int32_t *v, int64_t n_contacts, int32_t n_nodes,
            const orc_params *p, int32_t *counts, uint8_t *node_states);

/* Countdown classification used for the summary/node CSVs. */
int orc_countdown_class(int32_t c, int32_t exposed, int32_t infectious,
                        int32_t resistant);

#ifdef __cplusplus
}
#endif
#endif
