/* Built and run by tests/test_capi_cpu.py without a GPU: include/maxmulsk.h
 * compiles as plain C99 (and as C++), every entry point it declares links
 * against libmaxmulsk_b200.so, and the host-only calls behave -- the check a
 * C caller of the reference's capi/maxmulsk.h would make after swapping the
 * include path and the library. */
#include <stdio.h>
#include <string.h>

#include "maxmulsk.h"

typedef void (*entry_fn)(void);

int main(void) {
    /* Every declared entry point resolves at link time. */
    const entry_fn entries[] = {
        (entry_fn)maxmulsk_sgemm_v3, (entry_fn)maxmulsk_sgemm_v4, (entry_fn)maxmulsk_sgemm_v3_dev,
        (entry_fn)maxmulsk_sgemm_v4_dev, (entry_fn)maxmulsk_classify, (entry_fn)maxmulsk_choose,
        (entry_fn)maxmulsk_choose_rule, (entry_fn)maxmulsk_workspace_bytes, (entry_fn)maxmulsk_sgemm_plan_dev,
        (entry_fn)maxmulsk_sgemm_plan, (entry_fn)maxmulsk_sgemm_split, (entry_fn)maxmulsk_sgemm_split_dev,
        (entry_fn)maxmulsk_probe_split_bytes, (entry_fn)maxmulsk_probe_split_dev,
        (entry_fn)maxmulsk_probe_timeout_dev, (entry_fn)maxmulsk_grouped_create, (entry_fn)maxmulsk_grouped_launch,
        (entry_fn)maxmulsk_grouped_info, (entry_fn)maxmulsk_grouped_destroy, (entry_fn)maxmulsk_sgemm_grouped_dev,
        (entry_fn)maxmulsk_candidates, (entry_fn)maxmulsk_autotune_time_dev, (entry_fn)maxmulsk_autotune_dev,
        (entry_fn)maxmulsk_tuning_load, (entry_fn)maxmulsk_tuning_save, (entry_fn)maxmulsk_tuning_clear,
        (entry_fn)maxmulsk_model_load, (entry_fn)maxmulsk_mlp_features, (entry_fn)maxmulsk_mlp_predict_host,
        (entry_fn)maxmulsk_mlp_forward_dev, (entry_fn)maxmulsk_mlp_backward_dev, (entry_fn)maxmulsk_mlp_adam_dev,
        (entry_fn)maxmulsk_mlp_predict_dev, (entry_fn)maxmulsk_sgemm_plan_static_dev,
        (entry_fn)maxmulsk_stream_status, (entry_fn)maxmulsk_status_string, (entry_fn)maxmulsk_last_error_message,
        (entry_fn)maxmulsk_version, (entry_fn)maxmulsk_phase_timing, (entry_fn)maxmulsk_phase_report,
    };
    for (size_t i = 0; i < sizeof entries / sizeof entries[0]; i++)
        if (!entries[i]) return 10;

    /* Plan validation and sizing (capi/maxmulsk.h has none; the v4 classify rule). */
    maxmulsk_plan p;
    memset(&p, 0, sizeof p);
    p.precision = MAXMULSK_PREC_FP32;
    p.tile_m = 128;
    p.tile_n = 128;
    p.split_k = 1;
    if (maxmulsk_classify(256, 256, 256, &p) != MAXMULSK_OK) return 11;
    p.tile_n = 96;
    if (maxmulsk_classify(256, 256, 256, &p) == MAXMULSK_OK) return 12;

    /* Empty shapes (capi/maxmulsk.cpp:13-20): OK, C untouched. */
    float C[4] = {3.75f, 3.75f, 3.75f, 3.75f};
    if (maxmulsk_sgemm_v3(NULL, NULL, C, 0, 4, 4) != MAXMULSK_OK) return 13;
    if (maxmulsk_sgemm_v4(NULL, NULL, C, 4, 4, 0) != MAXMULSK_OK) return 14;
    for (int i = 0; i < 4; i++)
        if (C[i] != 3.75f) return 15;

    /* Status names and the phase report with nothing recorded. */
    if (strcmp(maxmulsk_status_string(MAXMULSK_OK), maxmulsk_status_string(MAXMULSK_ERR_TIMEOUT)) == 0) return 16;
    char report[MAXMULSK_PHASE_REPORT_BYTES];
    if (maxmulsk_phase_report(report, sizeof report) != 2 || strcmp(report, "{}") != 0) return 17;

    printf("c-abi ok %s\n", maxmulsk_version());
    return 0;
}
