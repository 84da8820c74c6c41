// Entry points whose implementation lands in pipeline.cu / server.cu.
#include "engine.cuh"
extern "C" {
phr_status phr_index_create(phr_ctx*, const uint8_t*, uint64_t, const phr_sketch*, phr_alphabet, phr_index**) { return PHR_ERR_STATE; }
void phr_index_destroy(phr_index*) {}
phr_status phr_index_get_info(const phr_index*, phr_index_info*) { return PHR_ERR_STATE; }
phr_status phr_sketch_batch(phr_ctx*, const phr_seq_batch*, int32_t, int32_t, phr_alphabet, const uint64_t*, uint64_t*, uint32_t*, uint32_t*) { return PHR_ERR_STATE; }
phr_status phr_seed_chain_batch(phr_ctx*, const phr_index*, const phr_sketch*, uint64_t, phr_chain_arena*) { return PHR_ERR_STATE; }
phr_status phr_align_reads(phr_ctx*, const phr_index*, const phr_read_batch*, const phr_align_config*, phr_read_result_arena*, phr_align_stats*) { return PHR_ERR_STATE; }
phr_status phr_server_create(phr_ctx*, const phr_index*, const phr_server_config*, phr_server**) { return PHR_ERR_STATE; }
phr_status phr_server_submit(phr_server*, const uint8_t*, uint32_t, uint64_t*) { return PHR_ERR_STATE; }
phr_status phr_server_poll(phr_server*, phr_server_result*, uint32_t, phr_alignment*, uint64_t, char*, uint64_t, uint32_t, uint32_t*) { return PHR_ERR_STATE; }
phr_status phr_server_destroy(phr_server*) { return PHR_ERR_STATE; }
}
