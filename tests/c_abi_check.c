/* A plain C caller of libgaffa_b200 (no Python, no torch): builds the riptide
 * FFA plan of the plain end-to-end workload (2^18 samples at 64 us, periods
 * 0.2-2 s, bins 180-256) through the two-call pattern, checks an argument
 * error and its message, and prints the plan for tests/test_c_abi_program.py
 * to compare with the Python binding.  Host-only entry points: runs without
 * a GPU. */
#include <stdio.h>
#include <stdlib.h>
#include "gaffa_b200.h"

int main(void) {
  gf_plan_options o;
  o.period_min = 0.2;
  o.period_max = 2.0;
  o.bins_min = 180;
  o.bins_max = 256;
  o.min_periods = 1;
  o.duty_cycle_max = 0.2;
  o.width_trial_spacing = 1.5;
  o.max_tasks = 1000000;
  uint64_t ntasks = 0, nwidths = 0;
  if (gf_make_riptide_ffa_plan(1u << 18, 64e-6, &o, NULL, 0, &ntasks, NULL, 0, &nwidths) != GF_OK) {
    fprintf(stderr, "sizing call failed: %s\n", gf_last_error());
    return 1;
  }
  gf_ffa_task* tasks = (gf_ffa_task*)calloc(ntasks, sizeof(gf_ffa_task));
  uint64_t* widths = (uint64_t*)calloc(nwidths, sizeof(uint64_t));
  if (gf_make_riptide_ffa_plan(1u << 18, 64e-6, &o, tasks, ntasks, &ntasks, widths, nwidths, &nwidths) != GF_OK) {
    fprintf(stderr, "plan call failed: %s\n", gf_last_error());
    return 1;
  }
  printf("tasks %llu widths %llu\n", (unsigned long long)ntasks, (unsigned long long)nwidths);
  for (uint64_t i = 0; i < ntasks; i += ntasks / 5 ? ntasks / 5 : 1)
    printf("task %llu bins %llu rows %llu rows_eval %llu factor %.17g\n", (unsigned long long)i,
           (unsigned long long)tasks[i].bins, (unsigned long long)tasks[i].rows,
           (unsigned long long)tasks[i].rows_eval, tasks[i].downsample_factor);
  /* batched launches and the copy-ring status: null arguments are
     rejected before any CUDA call */
  gf_preprocess_batch* pb = NULL;
  int bad = 0;
  bad |= gf_preprocess_batch_create(NULL, 1, 0, &pb) != GF_EINVAL;
  bad |= gf_preprocess_batch_run(NULL, NULL) != GF_EINVAL;
  bad |= gf_ffa_batch_prepare_all(NULL, NULL) != GF_EINVAL;
  bad |= gf_ffa_batch_bind_series(NULL, NULL, NULL, NULL) != GF_EINVAL;
  bad |= gf_dedisp_check(NULL, NULL) != GF_EINVAL;
  printf("batched entry points reject null arguments: %s\n", bad ? "no" : "yes");
  uint64_t n = 0;
  const int rc = gf_downsampled_size(100, 0.5, &n); /* factor < 1: rejected */
  printf("error %d %s\n", rc, gf_last_error());
  free(tasks);
  free(widths);
  return rc == GF_EINVAL && !bad ? 0 : 2;
}
