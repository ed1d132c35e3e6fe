/* `replay` -- drop-in replacement of the reference executable
 * (tool/gpu_cpu_temporal_sim.cu:570-1185) on top of libreplay.
 *
 * Same flags, defaults, exit codes and CSV outputs:
 *   replay <graph file> [--M n] [--step-size s] [--iterations k]
 *          [--summary-out f] [--node-state-out f] [--initial-infected p]
 *          [--infect-prob p] [--exposed-duration s] [--infectious-duration s]
 *          [--resistant-duration s] [--start-time t]
 *          [--static-network-duration s | --time-step s]
 *          [--cpu-only] [--cpu-threads n] [-q | --disable-debug-prints]
 * Output files are deleted and truncated while the flags are read; the
 * summary CSV is `time,simulation_id,exposed,infectious,resistant,
 * susceptible` with one row per replica per time, the first two times both
 * equal to the start time (the initial state and the end of iteration 1).
 * The node CSV is `time,simulation_id,node_id,state` with compressed node
 * indices.  --cpu-only and --cpu-threads are accepted for compatibility; the
 * replay always runs on the GPU.
 *
 * Additive flags (new modes): --transition countdown|geometric, --seed n,
 * --initial-count k, --beta b, --p-ei p, --p-ir p, --p-rs p, --no-exposed,
 * --sis, --path auto|plain|batched, --csr per-step|prebuilt, --ncls-cap 0|1,
 * --device d.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/replay.h"

static FILE *g_node_fp = NULL;

static char *fmt_i64(char *p, int64_t v) {
  char tmp[24];
  int n = 0;
  uint64_t u = v < 0 ? (uint64_t)(-(v + 1)) + 1 : (uint64_t)v;
  if (v < 0) *p++ = '-';
  do {
    tmp[n++] = (char)('0' + u % 10);
    u /= 10;
  } while (u);
  while (n) *p++ = tmp[--n];
  return p;
}

/* Node-state lines arrive formatted by the device (rp_sim_run_text). */
static int node_text_cb(void *user, int32_t step_index, int64_t ts, const char *text, size_t len) {
  (void)user;
  (void)step_index;
  (void)ts;
  if (!g_node_fp) return 0;
  return fwrite(text, 1, len, g_node_fp) == len ? 0 : 1;
}

static void usage(const char *argv0) {
  fprintf(stderr, "Usage: %s <graph file> [options]\n", argv0);
  fprintf(stderr, "Options:\n");
  fprintf(stderr, "  --cpu-only             Accepted for compatibility (runs on the GPU).\n");
  fprintf(stderr, "  --cpu-threads <int>    Accepted for compatibility.\n");
  fprintf(stderr, "  --M <int>              Number of parallel simulations.\n");
  fprintf(stderr, "  --step-size <float>    Time step size.\n");
  fprintf(stderr, "  --iterations <int>     Number of main simulation steps.\n");
  fprintf(stderr, "  --summary-out <file>   Output file for summary state counts.\n");
  fprintf(stderr, "  --node-state-out <file> Output file for per-node states.\n");
  fprintf(stderr, "  --initial-infected <float>     Initial infection probability [0-1]\n");
  fprintf(stderr, "  --infect-prob <float>          Infection prob if exposed [0-1]\n");
  fprintf(stderr, "  --exposed-duration <int>       Duration (seconds) before an infected person becomes infectious\n");
  fprintf(stderr, "  --infectious-duration <int>    Duration (seconds) a person remains infectious before recovery\n");
  fprintf(stderr, "  --resistant-duration <int>     Duration (seconds) a recovered person remains resistant before becoming susceptible again\n");
  fprintf(stderr, "  --start-time <epoch>         Unix start time of the simulation.\n");
  fprintf(stderr, "  --static-network-duration <seconds>  Duration (seconds) of each static contact network window.\n");
  fprintf(stderr, "  [deprecated] --time-step <seconds>   Alias for --static-network-duration.\n");
  fprintf(stderr, "  --transition countdown|geometric   Transition rule (default countdown).\n");
  fprintf(stderr, "  --seed <int>  --initial-count <int>  --beta <float>  --p-ei/--p-ir/--p-rs <float>\n");
  fprintf(stderr, "  --no-exposed  --sis  --path auto|plain|batched  --csr per-step|prebuilt\n");
  fprintf(stderr, "  --ncls-cap 0|1  --device <int>\n");
}

int main(int argc, char **argv) {
  printf("=== GPU-Accelerated Temporal Epidemiology Simulation ===\n");
  if (argc < 2) {
    usage(argv[0]);
    return 1;
  }
  for (int i = 1; i < argc; ++i) {
    if (strcmp(argv[i], "--disable-debug-prints") == 0 || strcmp(argv[i], "-q") == 0) {
      if (!freopen("/dev/null", "w", stdout)) return 1;
      break;
    }
  }
  rp_params p;
  rp_params_default(&p);
  const char *filename = NULL;
  FILE *summary_fp = NULL;
  int device = 0;
  for (int i = 1; i < argc; ++i) {
    const char *a = argv[i];
    const int has = i + 1 < argc;
    if (a[0] != '-') {
      filename = a;
      continue;
    }
    if (strcmp(a, "--cpu-only") == 0) {
      fprintf(stderr, "[INFO] --cpu-only: this build runs the replay on the GPU.\n");
    } else if (strcmp(a, "--disable-debug-prints") == 0 || strcmp(a, "-q") == 0) {
    } else if (strcmp(a, "--cpu-threads") == 0 && has) {
      ++i;
    } else if (strcmp(a, "--M") == 0 && has) {
      p.n_replicas = atoi(argv[++i]);
    } else if (strcmp(a, "--step-size") == 0 && has) {
      p.step_size = (float)atof(argv[++i]);
    } else if (strcmp(a, "--iterations") == 0 && has) {
      p.n_steps = atoi(argv[++i]);
    } else if (strcmp(a, "--summary-out") == 0 && has) {
      remove(argv[i + 1]);
      summary_fp = fopen(argv[++i], "w");
      if (!summary_fp) {
        fprintf(stderr, "Error: Could not open summary output file.\n");
        return 1;
      }
    } else if (strcmp(a, "--node-state-out") == 0 && has) {
      remove(argv[i + 1]);
      g_node_fp = fopen(argv[++i], "w");
      if (!g_node_fp) {
        fprintf(stderr, "Error: Could not open node state output file.\n");
        return 1;
      }
    } else if (strcmp(a, "--initial-infected") == 0 && has) {
      p.initial_infected = (float)atof(argv[++i]);
    } else if (strcmp(a, "--infect-prob") == 0 && has) {
      p.infect_prob = (float)atof(argv[++i]);
    } else if (strcmp(a, "--exposed-duration") == 0 && has) {
      p.exposed_duration = atoi(argv[++i]);
    } else if (strcmp(a, "--infectious-duration") == 0 && has) {
      p.infectious_duration = atoi(argv[++i]);
    } else if (strcmp(a, "--resistant-duration") == 0 && has) {
      p.resistant_duration = atoi(argv[++i]);
    } else if (strcmp(a, "--start-time") == 0 && has) {
      p.start_time = (int64_t)atoll(argv[++i]);
    } else if ((strcmp(a, "--static-network-duration") == 0 ||
                strcmp(a, "--time-step") == 0) && has) {
      p.window = (int64_t)atoll(argv[++i]);
    } else if (strcmp(a, "--transition") == 0 && has) {
      const char *v = argv[++i];
      if (strcmp(v, "countdown") == 0)
        p.transition = RP_TRANSITION_COUNTDOWN;
      else if (strcmp(v, "geometric") == 0)
        p.transition = RP_TRANSITION_GEOMETRIC;
      else {
        fprintf(stderr, "Unrecognized transition: %s\n", v);
        return 1;
      }
    } else if (strcmp(a, "--seed") == 0 && has) {
      p.seed = (uint64_t)strtoull(argv[++i], NULL, 10);
    } else if (strcmp(a, "--initial-count") == 0 && has) {
      p.initial_count = atoi(argv[++i]);
    } else if (strcmp(a, "--beta") == 0 && has) {
      p.beta = (float)atof(argv[++i]);
    } else if (strcmp(a, "--p-ei") == 0 && has) {
      p.p_ei = (float)atof(argv[++i]);
    } else if (strcmp(a, "--p-ir") == 0 && has) {
      p.p_ir = (float)atof(argv[++i]);
    } else if (strcmp(a, "--p-rs") == 0 && has) {
      p.p_rs = (float)atof(argv[++i]);
    } else if (strcmp(a, "--no-exposed") == 0) {
      p.has_exposed = 0;
    } else if (strcmp(a, "--sis") == 0) {
      p.ir_to_s = 1;
    } else if (strcmp(a, "--path") == 0 && has) {
      const char *v = argv[++i];
      p.path = strcmp(v, "plain") == 0 ? RP_PATH_PLAIN
               : strcmp(v, "batched") == 0 ? RP_PATH_BATCHED
                                           : RP_PATH_AUTO;
    } else if (strcmp(a, "--csr") == 0 && has) {
      p.csr_mode = strcmp(argv[++i], "prebuilt") == 0 ? RP_CSR_PREBUILT : RP_CSR_PER_STEP;
    } else if (strcmp(a, "--ncls-cap") == 0 && has) {
      p.ncls_cap = atoi(argv[++i]) != 0;
    } else if (strcmp(a, "--device") == 0 && has) {
      device = atoi(argv[++i]);
    } else {
      fprintf(stderr, "Unrecognized option: %s\n", a);
      return 1;
    }
  }
  if (!filename) {
    fprintf(stderr, "Missing contact network file argument.\n");
    return 1;
  }
  if (summary_fp)
    fprintf(summary_fp, "time,simulation_id,exposed,infectious,resistant,susceptible\n");
  if (g_node_fp) fprintf(g_node_fp, "time,simulation_id,node_id,state\n");

  rp_graph *g = NULL;
  if (rp_graph_load_text(filename, device, &g) != RP_OK) {
    fprintf(stderr, "%s\n", rp_last_error());
    fprintf(stderr, "No intervals read or parse error.\n");
    return 1;
  }
  rp_graph_info gi;
  rp_graph_get_info(g, &gi);
  printf("[INFO] Node count set from NODE_LIST: %d\n", gi.n_nodes);
  fprintf(stderr, "Parsed %lld edges (intervals) from graph.\n", (long long)gi.n_contacts);
  fprintf(stderr, "Interval index built. nlists=%lld, duration classes=%d.\n",
          (long long)gi.nlists, gi.n_classes);

  p.record_node_states = g_node_fp != NULL;
  rp_sim *s = NULL;
  if (rp_sim_create(g, &p, &s) != RP_OK) {
    fprintf(stderr, "Error: %s\n", rp_last_error());
    rp_graph_free(g);
    return 1;
  }
  printf("\nStarting temporal Monte Carlo simulation for %d iterations...\n", p.n_steps);
  printf("[INFO] Simulation start time: %lld, time step: %.3f seconds, static network "
         "window: %lld seconds\n",
         (long long)p.start_time, (double)p.step_size, (long long)p.window);
  /* Callers time the simulation phase from the moment this marker arrives
   * on a pipe (the scaling benchmark scripts under replay/scaling), so it is
   * not left in the stdio buffer until the end. */
  fflush(stdout);
  const int32_t M = p.n_replicas, T = p.n_steps;
  int32_t *counts = (int32_t *)malloc(sizeof(int32_t) * (size_t)(T + 1) * (size_t)M * 4);
  int64_t *ts = (int64_t *)malloc(sizeof(int64_t) * (size_t)(T + 1));
  if (!counts || !ts) {
    fprintf(stderr, "Error: unable to allocate host arrays.\n");
    return 1;
  }
  const rp_status run_st = g_node_fp ? rp_sim_run_text(s, counts, node_text_cb, NULL)
                                     : rp_sim_run(s, counts, NULL, NULL);
  if (run_st != RP_OK) {
    fprintf(stderr, "Error: %s\n", rp_last_error());
    return 1;
  }
  rp_sim_timestamps(s, ts);
  for (int32_t t = 0; t < T; ++t)
    printf("\n--- Iteration %d (sim time %lld) ---\n", t + 1, (long long)ts[t + 1]);
  if (summary_fp) {
    size_t cap = 1 << 22;
    char *buf = (char *)malloc(cap);
    char *q = buf;
    for (int32_t t = 0; t <= T; ++t)
      for (int32_t r = 0; r < M; ++r) {
        if ((size_t)(q - buf) + 128 > cap) {
          fwrite(buf, 1, (size_t)(q - buf), summary_fp);
          q = buf;
        }
        const int32_t *c = counts + ((int64_t)t * M + r) * 4;
        q = fmt_i64(q, ts[t]);
        *q++ = ',';
        q = fmt_i64(q, r);
        for (int k = 0; k < 4; ++k) {
          *q++ = ',';
          q = fmt_i64(q, c[k]);
        }
        *q++ = '\n';
      }
    fwrite(buf, 1, (size_t)(q - buf), summary_fp);
    free(buf);
    fclose(summary_fp);
  }
  if (g_node_fp) fclose(g_node_fp);
  printf("Simulation done.\n");
  free(counts);
  free(ts);
  rp_sim_free(s);
  rp_graph_free(g);
  return 0;
}
