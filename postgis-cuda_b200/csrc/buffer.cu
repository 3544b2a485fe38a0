// Distance and negative-buffer joins (engine/buffer.cuh of the reference). Filled in below.
#include "engine.h"
namespace gsj {
void dwithin_host(gsj_ctx*, const gsj_layer*, const gsj_layer*, double, int, const gsj_join_opts*, gsj_pairs_sink, void*, gsj_join_stats*) {
  throw Error(GSJ_ERR_ARG, "dwithin: not built yet");
}
void erode_host(gsj_ctx*, const gsj_layer*, const gsj_layer*, double, double, int, const uint8_t*, const gsj_join_opts*, gsj_pairs_sink, void*,
                gsj_join_stats*) {
  throw Error(GSJ_ERR_ARG, "erode: not built yet");
}
void points_buffer_host(gsj_ctx*, const gsj_layer*, const gsj_layer*, double, int, const gsj_join_opts*, gsj_pairs_sink, void*, gsj_join_stats*) {
  throw Error(GSJ_ERR_ARG, "points buffer: not built yet");
}
}  // namespace gsj
