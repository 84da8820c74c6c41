// A C++ caller of the C ABI, as a non-Python host would bind it: reads pairs from a
// text file (one "query target" pair per line), runs phr_extend_batch for the engine
// given on the command line, and prints "status ed qs qe ts te cigar" per pair.
// Usage: extend_harness <engine 0..3> <pairs.txt>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/phraya_gpu.h"

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <engine> <pairs.txt>\n", argv[0]);
        return 2;
    }
    const int engine = std::atoi(argv[1]);
    std::ifstream in(argv[2]);
    std::string line, seq;
    std::vector<uint64_t> q_off, t_off;
    std::vector<uint32_t> q_len, t_len;
    while (std::getline(in, line)) {
        std::istringstream ss(line);
        std::string q, t;
        ss >> q >> t;
        if (q == "-") q.clear();
        if (t == "-") t.clear();
        q_off.push_back(seq.size());
        q_len.push_back(static_cast<uint32_t>(q.size()));
        seq += q;
        t_off.push_back(seq.size());
        t_len.push_back(static_cast<uint32_t>(t.size()));
        seq += t;
    }
    const uint64_t n = q_off.size();
    uint64_t bound = 16;
    for (uint64_t i = 0; i < n; ++i) bound += PHR_CIGAR_BOUND(q_len[i], t_len[i]);
    phr_pair_batch b{n, reinterpret_cast<const uint8_t*>(seq.data()), seq.size(), q_off.data(), q_len.data(),
                     t_off.data(), t_len.data(), nullptr, nullptr};
    std::vector<phr_alignment> aln(n);
    std::vector<char> cig(bound);
    phr_result_arena out{aln.data(), cig.data(), bound, 0};
    phr_ctx* ctx = nullptr;
    phr_status st = phr_ctx_create(0, nullptr, &ctx);
    if (st != PHR_OK) {
        std::fprintf(stderr, "phr_ctx_create: %s\n", phr_status_string(st));
        return 1;
    }
    phr_affine_costs costs{4, 6, 2};
    st = phr_extend_batch(ctx, static_cast<phr_engine>(engine), &b, costs, &out);
    if (st != PHR_OK) {
        std::fprintf(stderr, "phr_extend_batch: %s (%s)\n", phr_status_string(st), phr_ctx_last_error(ctx));
        phr_ctx_destroy(ctx);
        return 1;
    }
    for (uint64_t i = 0; i < n; ++i) {
        const phr_alignment& a = aln[i];
        std::printf("%d %u %u %u %u %u %.*s\n", a.status, a.edit_distance, a.query_start, a.query_end,
                    a.target_start, a.target_end, static_cast<int>(a.cigar_len), cig.data() + a.cigar_off);
    }
    phr_ctx_destroy(ctx);
    return 0;
}
