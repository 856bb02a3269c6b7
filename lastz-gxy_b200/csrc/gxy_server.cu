// gxy_server.cu -- serving loop (placeholder until the loop lands).
#include "gxy_engine.cuh"

extern "C" {
gxy_status gxy_server_create(gxy_ctx*, uint32_t, const gxy_table* const*, const gxy_search_params*,
                             const gxy_server_opts*, gxy_server**) {
    return GXY_EUNSUPPORTED;
}
gxy_status gxy_server_submit(gxy_server*, uint32_t, const gxy_packed_seq*, uint64_t*) { return GXY_EUNSUPPORTED; }
gxy_status gxy_server_wait(gxy_server*, uint64_t, uint32_t, gxy_hsp_buf*, gxy_hsp_buf*, double*) {
    return GXY_EUNSUPPORTED;
}
gxy_status gxy_server_get_stats(gxy_server*, gxy_server_stats*) { return GXY_EUNSUPPORTED; }
gxy_status gxy_server_destroy(gxy_server*) { return GXY_EUNSUPPORTED; }
}
