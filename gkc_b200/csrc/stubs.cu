// Entry points whose kernels are not in this build yet.
#include "ctx.h"

gkc_status gkc_server_create(int, uint64_t, int, gkc_server **) { return GKC_ERR_INTERNAL; }
void gkc_server_destroy(gkc_server *) {}
gkc_status gkc_server_submit(gkc_server *, const gkc_params *, const char *, const uint64_t *,
                             uint64_t, uint64_t *) { return GKC_ERR_INTERNAL; }
gkc_status gkc_server_submit_device_synth(gkc_server *, const gkc_params *, int, uint64_t, uint64_t,
                                          uint64_t *) { return GKC_ERR_INTERNAL; }
gkc_status gkc_server_poll(gkc_server *, uint64_t, gkc_job_info *) { return GKC_ERR_INTERNAL; }
gkc_status gkc_server_wait(gkc_server *, uint64_t, double, gkc_job_info *) { return GKC_ERR_INTERNAL; }
gkc_status gkc_server_cancel(gkc_server *, uint64_t) { return GKC_ERR_INTERNAL; }
gkc_status gkc_server_copy_result(gkc_server *, uint64_t, uint64_t *, uint64_t *, uint32_t *) {
  return GKC_ERR_INTERNAL;
}
gkc_status gkc_server_release(gkc_server *, uint64_t) { return GKC_ERR_INTERNAL; }
uint64_t gkc_job_hbm_estimate(const gkc_params *, uint64_t, uint64_t) { return 0; }
