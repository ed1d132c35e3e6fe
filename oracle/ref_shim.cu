// Function-level access to the reference implementation, for tests only.
//
// This translation unit compiles the reference's own simulation source
// (tool/gpu_cpu_temporal_sim.cu, included by path from the reference tree by
// oracle/Makefile) with its `main` renamed, and exports `extern "C"` wrappers
// around its file-static helpers so that tests can call them through ctypes:
//
//   ref_parse            -> parse_edgelist_build_intervals   (tool/temporal_contact_matrix.c:148-321)
//   ref_window_query     -> build_interval_db_wrapper + find_intervals with the
//                           driver's nbuf = nlists argument   (tool/gpu_cpu_temporal_sim.cu:973-991)
//   ref_build_csr        -> build_csr_from_intervals          (tool/gpu_cpu_temporal_sim.cu:238-350)
//   ref_cpu_spmm         -> CPUComputeSpMM (Eigen)            (tool/gpu_cpu_temporal_sim.cu:403-433)
//   ref_infection_prob   -> CPUComputeInfectionProbability    (tool/gpu_cpu_temporal_sim.cu:439-458)
//   ref_update_countdown -> CPUUpdateCountdownVector          (tool/gpu_cpu_temporal_sim.cu:489-500)
//   ref_infectious       -> CPUGenerateInfectiousVector       (tool/gpu_cpu_temporal_sim.cu:381-394)
//   ref_write_state      -> write_simulation_state            (tool/gpu_cpu_temporal_sim.cu:505-568)
//
// It is test infrastructure: nothing in the product links it.
#include <fcntl.h>
#include <unistd.h>

#define main replay_ref_main
#include "gpu_cpu_temporal_sim.cu"
#undef main

namespace {
struct StdoutMute {
  int saved = -1;
  explicit StdoutMute(bool on) {
    if (!on) return;
    fflush(stdout);
    saved = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) {
      dup2(devnull, 1);
      close(devnull);
    }
  }
  ~StdoutMute() {
    if (saved < 0) return;
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
  }
};
}  // namespace

extern "C" {

void ref_free(void *p) { free(p); }

// Parses a contact file with the reference parser.  Returns the number of
// intervals (or -1 on a parse failure); arrays are malloc'd and owned by the
// caller (ref_free).  `n_nodes` receives the NODE_LIST token count.
int ref_parse(const char *path, int quiet, int *n_nodes, int64_t **start,
              int64_t **end, int32_t **src, int32_t **tgt) {
  StdoutMute mute(quiet != 0);
  int count = 0;
  IntervalMap *im = parse_edgelist_build_intervals(path, &count);
  *n_nodes = get_total_node_count();
  if (!im) {
    free_node_map();
    return -1;
  }
  *start = (int64_t *)malloc(sizeof(int64_t) * (count > 0 ? count : 1));
  *end = (int64_t *)malloc(sizeof(int64_t) * (count > 0 ? count : 1));
  *src = (int32_t *)malloc(sizeof(int32_t) * (count > 0 ? count : 1));
  *tgt = (int32_t *)malloc(sizeof(int32_t) * (count > 0 ? count : 1));
  for (int i = 0; i < count; i++) {
    int s, t;
    unpack_node_pair(im[i].target_id, &s, &t);
    (*start)[i] = im[i].start;
    (*end)[i] = im[i].end;
    (*src)[i] = s;
    (*tgt)[i] = t;
  }
  free(im);
  free_node_map();
  return count;
}

// Builds the NCLS over the given contacts and runs the reference main loop's
// per-step query for [ws, we).  Hit buffers must hold `n` entries.  Returns
// the number of hits that loop would pass to build_csr_from_intervals.
int ref_window_query(const int64_t *start, const int64_t *end,
                     const int32_t *src, const int32_t *tgt, int n, int64_t ws,
                     int64_t we, int *out_nlists, int *out_ncompact,
                     int64_t *hit_start, int64_t *hit_end, int32_t *hit_src,
                     int32_t *hit_tgt) {
  IntervalMap *im = interval_map_alloc(n);
  for (int i = 0; i < n; i++) {
    im[i].start = start[i];
    im[i].end = end[i];
    im[i].target_id = pack_node_pair(src[i], tgt[i]);
    im[i].sublist = -1;
  }
  IntervalDBWrapper dbw;
  if (!build_interval_db_wrapper(im, n, &dbw)) {
    free(im);
    return -1;
  }
  *out_nlists = dbw.nlists;
  *out_ncompact = dbw.n;
  IntervalMap *hits = (IntervalMap *)malloc(
      sizeof(IntervalMap) * (dbw.nlists > 0 ? dbw.nlists : dbw.n));
  IntervalIterator *it = interval_iterator_alloc();
  int n_return = 0;
  find_intervals(it, ws, we, dbw.im, dbw.n, dbw.subheader, dbw.nlists, hits,
                 dbw.nlists, &n_return, &it);
  free_interval_iterator(it);
  for (int i = 0; i < n_return; i++) {
    int s, t;
    unpack_node_pair(hits[i].target_id, &s, &t);
    hit_start[i] = hits[i].start;
    hit_end[i] = hits[i].end;
    hit_src[i] = s;
    hit_tgt[i] = t;
  }
  free(hits);
  free_interval_db_wrapper(&dbw);
  return n_return;
}

// Runs build_csr_from_intervals on explicit hits.  row_ptr holds n_nodes+1,
// col/val hold 2*n_hits entries.  Returns nnz.
long ref_build_csr(const int64_t *hit_start, const int64_t *hit_end,
                   const int32_t *hit_src, const int32_t *hit_tgt, int n_hits,
                   int n_nodes, int64_t ws, int64_t we, float weight_scale,
                   int32_t *row_ptr, int32_t *col, float *val) {
  IntervalMap *hits = (IntervalMap *)malloc(sizeof(IntervalMap) *
                                            (n_hits > 0 ? n_hits : 1));
  for (int i = 0; i < n_hits; i++) {
    hits[i].start = hit_start[i];
    hits[i].end = hit_end[i];
    hits[i].target_id = pack_node_pair(hit_src[i], hit_tgt[i]);
    hits[i].sublist = -1;
  }
  int *rp = NULL, *ci = NULL;
  float *cv = NULL;
  size_t nnz = 0;
  build_csr_from_intervals(hits, n_hits, n_nodes, &rp, &ci, &cv, &nnz, ws, we,
                           weight_scale);
  memcpy(row_ptr, rp, sizeof(int) * (size_t)(n_nodes + 1));
  if (nnz) {
    memcpy(col, ci, sizeof(int) * nnz);
    memcpy(val, cv, sizeof(float) * nnz);
  }
  free(rp);
  free(ci);
  free(cv);
  free(hits);
  return (long)nnz;
}

void ref_cpu_spmm(const int32_t *row_ptr, const int32_t *col, const float *val,
                  long nnz, int n, const float *infectious, float *exposure,
                  int m) {
  CPUComputeSpMM(row_ptr, col, val, (size_t)nnz, n, infectious, exposure, m);
}

void ref_set_durations(int exposed, int infectious, int resistant,
                       float infect_prob) {
  gExposedDuration = exposed;
  gInfectiousDuration = infectious;
  gResistantDuration = resistant;
  gUpperRange = exposed + infectious + resistant;
  gMediumRange = infectious + resistant;
  gLowerRange = resistant;
  gSusceptibleInfectProb = infect_prob;
}

void ref_infectious(const int32_t *countdown, float *infectious, int n, int m) {
  CPUGenerateInfectiousVector(countdown, infectious, n, m);
}

void ref_infection_prob(float *exposure, const int32_t *countdown, int n,
                        int m, float step) {
  CPUComputeInfectionProbability(exposure, countdown, n, m, step);
}

void ref_update_countdown(int32_t *countdown, int n, int m, float step) {
  CPUUpdateCountdownVector(countdown, n, m, step);
}

// Appends write_simulation_state rows for one timestamp to the given files
// (either path may be NULL).
int ref_write_state(const char *summary_path, const char *node_path,
                    const int32_t *countdown, int n, int m, int64_t ts) {
  FILE *sf = summary_path ? fopen(summary_path, "a") : NULL;
  FILE *nf = node_path ? fopen(node_path, "a") : NULL;
  if ((summary_path && !sf) || (node_path && !nf)) return -1;
  write_simulation_state(sf, nf, countdown, n, m, ts);
  if (sf) fclose(sf);
  if (nf) fclose(nf);
  return 0;
}

}  // extern "C"
