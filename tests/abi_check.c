/* C-language check of the drop-in boundary: include/diablo_b200.h compiles
 * as strict C99 and every entry it declares resolves in libdiablo_b200.so
 * (the link fails otherwise).  Runs without a GPU: it calls only the entries
 * whose answer needs no device (version, argument errors, db_init failing
 * cleanly when no device is present or the arguments are bad).
 * Built and run by tests/test_host.py. */
#include <stdio.h>
#include <string.h>

#include "diablo_b200.h"

typedef void (*entry)(void);

int main(void) {
  /* every declared entry, referenced so the linker must resolve it */
  const entry all[] = {
      (entry)db_abi_version, (entry)db_last_error, (entry)db_init, (entry)db_finalize,
      (entry)db_upload_state, (entry)db_download_state, (entry)db_upload_field, (entry)db_download_field,
      (entry)db_set_clock, (entry)db_get_status, (entry)db_clear_status, (entry)db_fft_xz_to_fourier, (entry)db_fft_xz_to_fourier_dev,
      (entry)db_fft_xz_to_physical, (entry)db_fft_xz_to_physical_dev, (entry)db_rk_substep, (entry)db_rk_steps, (entry)db_rem_div,
      (entry)db_apply_bc_vel_post, (entry)db_courant, (entry)db_divergence, (entry)db_stats, (entry)db_budget, (entry)db_bpe, (entry)db_bin_ystar, (entry)db_les_stats, (entry)db_poisson_p,
      (entry)db_rem_div_static, (entry)db_sgs_create, (entry)db_sgs_destroy, (entry)db_sgs_set,
      (entry)db_sgs_get, (entry)db_sgs_set_range, (entry)db_sgs_forward, (entry)db_sgs_gradient,
      (entry)db_sgs_train_step, (entry)db_sgs_gemm_check, (entry)db_set_sgs_net, (entry)db_les_eval,
      (entry)db_sgs_targets, (entry)db_ensemble_create, (entry)db_ensemble_steps, (entry)db_ensemble_destroy,
      (entry)db_ensemble_error, (entry)db_ensemble_set_batched, (entry)db_ensemble_info, (entry)db_autotune, (entry)db_get_tuning, (entry)db_set_tuning, (entry)db_set_timing, (entry)db_stage_times,
      (entry)db_kernel_launches, (entry)db_set_wait_limit,
  };
  const int n = (int)(sizeof all / sizeof all[0]);
  if (db_abi_version() != 1) {
    fprintf(stderr, "abi version %d\n", db_abi_version());
    return 1;
  }
  /* argument errors come back as codes, with a message, never an abort */
  db_ctx* ctx = NULL;
  if (db_init(NULL, NULL, NULL, &ctx) != DB_ERR_ARG || ctx != NULL) {
    fprintf(stderr, "db_init(NULL) did not return DB_ERR_ARG\n");
    return 1;
  }
  const char* msg = db_last_error(NULL);
  if (!msg || !strlen(msg)) {
    fprintf(stderr, "no error message after a failed db_init\n");
    return 1;
  }
  if (db_rk_substep(NULL, 1) != DB_ERR_ARG || db_stats(NULL, NULL) != DB_ERR_ARG) {
    fprintf(stderr, "NULL context not rejected\n");
    return 1;
  }
  printf("abi ok: %d entries, last error \"%s\"\n", n, msg);
  return 0;
}
