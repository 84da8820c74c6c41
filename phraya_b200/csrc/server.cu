// Serving loop entry points (placeholder until the serving runtime lands).
#include "engine.cuh"
extern "C" {
phr_status phr_server_create(phr_ctx*, const phr_index*, const phr_server_config*, phr_server**) { return PHR_ERR_STATE; }
phr_status phr_server_submit(phr_server*, const uint8_t*, uint32_t, uint64_t*) { return PHR_ERR_STATE; }
phr_status phr_server_poll(phr_server*, phr_server_result*, uint32_t, phr_alignment*, uint64_t, char*, uint64_t, uint32_t, uint32_t*) { return PHR_ERR_STATE; }
phr_status phr_server_destroy(phr_server*) { return PHR_ERR_STATE; }
}
