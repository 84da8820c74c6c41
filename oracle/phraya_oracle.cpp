// phraya_oracle.cpp -- CPU restatement of phraya-align's seed -> chain -> extend path.
//
// TEST INFRASTRUCTURE ONLY. This file is the bit-exactness oracle and the timed CPU
// baseline; only tests/, __graft_entry__.smoke() and bench.py's CPU legs load it.
// The product (phraya_b200/) never links or calls it.
//
// The reference is Rust and cannot be built in this environment (no cargo/rustc), so
// each function below restates one reference function literally -- same loops, same
// full-width wavefront storage, same tie-break order -- citing the file:line it follows
// (paths relative to the phraya repository root). Parity of this restatement is pinned
// by the reference's own known-answer tests and seeded property sweeps, ported under
// tests/ (see tests/golden/known_answers.json).
//
// The minimizer sketcher is the one exception: phraya uses the third-party crate
// simd-minimizers 2.3.1 (phraya-core/Cargo.toml; version named in
// docs/adr/0013-protein-space-alphabet-support.md:31; call site phraya-core/src/types.rs:
// 1848-1869), whose source is not in the reference tree. `sketch_seq` restates its
// published algorithm (see the comment there); no reference test pins minimizer values
// or positions, so parity at the sketching boundary is unpinned.

#include <emmintrin.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../include/phraya_gpu.h"

namespace {

// ---------------------------------------------------------------------------
// count_matching_prefix: wfa_simd.rs:52-61 dispatching to the SSE2 tier :67-90,
// scalar tail :123-130.
// ---------------------------------------------------------------------------
inline size_t lcp(const uint8_t* a, size_t an, const uint8_t* b, size_t bn) {
    size_t n = an < bn ? an : bn;
    size_t i = 0;
    while (i + 16 <= n) {
        __m128i va = _mm_loadu_si128(reinterpret_cast<const __m128i*>(a + i));
        __m128i vb = _mm_loadu_si128(reinterpret_cast<const __m128i*>(b + i));
        unsigned mask = static_cast<unsigned>(_mm_movemask_epi8(_mm_cmpeq_epi8(va, vb))) & 0xFFFFu;
        if (mask != 0xFFFFu) return i + static_cast<size_t>(__builtin_ctz(mask ^ 0xFFFFu));
        i += 16;
    }
    while (i < n && a[i] == b[i]) ++i;
    return i;
}

// compact_cigar: wfa_simd.rs:1200-1222 (run-length encode, "<count><op>").
std::string compact_cigar(const std::vector<char>& ops) {
    std::string out;
    if (ops.empty()) return out;
    char cur = ops[0];
    size_t count = 1;
    for (size_t i = 1; i < ops.size(); ++i) {
        if (ops[i] == cur) {
            ++count;
        } else {
            out += std::to_string(count);
            out.push_back(cur);
            cur = ops[i];
            count = 1;
        }
    }
    out += std::to_string(count);
    out.push_back(cur);
    return out;
}

constexpr int32_t UNSET = INT32_MIN;

struct Seq {
    const uint8_t* p;
    int32_t n;
};

// The `extend` closure of fill_wfa (wfa_simd.rs:252-262), shared by every WFA variant.
inline int32_t wfa_extend_diag(const Seq& q, const Seq& t, int32_t q_pos, int32_t k) {
    int32_t j = q_pos - k;
    if (q_pos < 0 || q_pos >= q.n || j < 0 || j >= t.n) return q_pos;
    return q_pos + static_cast<int32_t>(lcp(q.p + q_pos, q.n - q_pos, t.p + j, t.n - j));
}

// ---------------------------------------------------------------------------
// Linear WFA, literal restatement with full-width per-score history.
// ---------------------------------------------------------------------------
struct LinFrame {
    std::vector<int32_t> wf;
    std::vector<uint8_t> op;
};

// traceback_wfa (wfa_simd.rs:1044-1130) / traceback_wfa_with_tend (:959-1041): the two
// differ only in the starting target index, passed here as `t_end`.
std::string lin_traceback(const std::vector<LinFrame>& hist, const Seq& q, const Seq& t,
                          int32_t edit_dist, int32_t t_end) {
    const int32_t tn = t.n;
    std::vector<char> ops;
    int32_t qi = q.n, ti = t_end;
    int32_t k = qi - ti;
    int32_t s = edit_dist;
    while (qi > 0 || ti > 0) {
        if (s < 0) break;
        size_t ki = static_cast<size_t>(k + tn);
        if (s == 0) {
            while (qi > 0 && ti > 0) {
                ops.push_back('M');
                --qi;
                --ti;
            }
            break;
        }
        const std::vector<uint8_t>& wf_ops = hist[s].op;
        uint8_t op = ki < wf_ops.size() ? wf_ops[ki] : 0;
        const std::vector<int32_t>& prev = hist[s - 1].wf;
        int32_t pred_pos, pred_k;
        auto at = [&](int64_t pk) -> int32_t {
            return (pk >= 0 && static_cast<size_t>(pk) < prev.size()) ? prev[pk] : 0;
        };
        switch (op) {
            case 1: pred_pos = at(ki); pred_k = k; break;
            case 2: pred_pos = at(static_cast<int64_t>(k) - 1 + tn); pred_k = k - 1; break;
            case 3: pred_pos = at(static_cast<int64_t>(k) + 1 + tn); pred_k = k + 1; break;
            default: pred_pos = at(ki); pred_k = k; break;
        }
        int32_t edit_start = (op == 1 || op == 2) ? pred_pos + 1 : pred_pos;
        int32_t match_count = qi - edit_start;
        for (int32_t c = 0; c < match_count; ++c) {
            ops.push_back('M');
            --qi;
            --ti;
        }
        switch (op) {
            case 1: ops.push_back('X'); --qi; --ti; break;
            case 2: ops.push_back('D'); --qi; break;
            case 3: ops.push_back('I'); --ti; break;
            default: break;
        }
        k = pred_k;
        --s;
    }
    std::reverse(ops.begin(), ops.end());
    return compact_cigar(ops);
}

// One wavefront step s of fill_wfa / fill_wfa_fitting_impl (wfa_simd.rs:291-331 and
// :430-468, identical bodies). Candidates are tried in the order [mismatch, ins, del]
// and Rust's `max_by_key` keeps the LAST maximal one, so ties prefer del > ins > mm.
void lin_step(const LinFrame& prevf, LinFrame& next, const Seq& q, const Seq& t, int32_t s) {
    const int32_t qn = q.n, tn = t.n;
    const std::vector<int32_t>& prev = prevf.wf;
    int32_t lo = -std::min(s, tn);
    int32_t hi = std::min(s, qn);
    for (int32_t k = lo; k <= hi; ++k) {
        size_t ki = static_cast<size_t>(k + tn);
        int32_t best_pos = UNSET;
        uint8_t best_op = 0;
        bool have = false;
        auto consider = [&](int32_t p, uint8_t o) {
            if (p == UNSET) return;
            if (!have || p >= best_pos) {  // >= : last maximal element wins
                best_pos = p;
                best_op = o;
                have = true;
            }
        };
        if (ki < prev.size() && prev[ki] != UNSET) consider(prev[ki] + 1, 1);
        if (k > -tn) {
            size_t kp = static_cast<size_t>(k - 1 + tn);
            if (kp < prev.size() && prev[kp] != UNSET) consider(prev[kp] + 1, 2);
        }
        if (k < qn) {
            size_t kp = static_cast<size_t>(k + 1 + tn);
            if (kp < prev.size() && prev[kp] != UNSET) consider(prev[kp], 3);
        }
        if (!have) continue;
        int32_t j = best_pos - k;
        if (best_pos < 0 || best_pos > qn || j < 0 || j > tn) continue;
        next.wf[ki] = wfa_extend_diag(q, t, best_pos, k);
        next.op[ki] = best_op;
    }
}

// fill_wfa (wfa_simd.rs:231-345): global linear WFA. Returns (cigar, edit distance).
std::string fill_wfa(const Seq& q, const Seq& t, int32_t* ed_out) {
    const int32_t qn = q.n, tn = t.n;
    const size_t size = static_cast<size_t>(qn + tn + 1);
    std::vector<LinFrame> hist;
    LinFrame cur{std::vector<int32_t>(size, UNSET), std::vector<uint8_t>(size, 0)};
    cur.wf[tn] = wfa_extend_diag(q, t, 0, 0);
    const int32_t target_diag = qn - tn;
    const size_t target_idx = static_cast<size_t>(target_diag + tn);
    if (cur.wf[target_idx] == qn) {
        *ed_out = 0;
        return lin_traceback(hist, q, t, 0, tn);
    }
    hist.push_back(std::move(cur));
    const int32_t max_s = qn + tn;
    for (int32_t s = 1; s <= max_s; ++s) {
        LinFrame next{std::vector<int32_t>(size, UNSET), std::vector<uint8_t>(size, 0)};
        lin_step(hist[s - 1], next, q, t, s);
        bool done = target_idx < next.wf.size() && next.wf[target_idx] >= qn;
        hist.push_back(std::move(next));
        if (done) {
            *ed_out = s;
            return lin_traceback(hist, q, t, s, tn);
        }
    }
    *ed_out = 0;  // wfa_simd.rs:343-344 fallback, unreachable for valid input
    return std::string();
}

// fitting_end_k (wfa_simd.rs:940-955): smallest k (largest t_end) with wf[k] >= qn.
bool fitting_end_k(const std::vector<int32_t>& wf, int32_t qn, int32_t tn, int32_t* t_end) {
    bool found = false;
    int32_t best = 0;
    for (int32_t k = qn - tn; k <= qn; ++k) {
        int32_t te = qn - k;
        if (te < 0 || te > tn) continue;
        size_t ki = static_cast<size_t>(k + tn);
        if (ki >= wf.size()) continue;
        if (wf[ki] >= qn) {
            if (!found || te > best) {
                best = te;
                found = true;
            }
        }
    }
    *t_end = best;
    return found;
}

// fill_wfa_fitting_impl (wfa_simd.rs:360-482). Returns false when abandoned (cap).
// max_s_cap < 0 means "no cap".
bool fill_wfa_fitting_impl(const Seq& q, const Seq& t, int64_t max_s_cap, std::string* cigar,
                           int32_t* ed, int32_t* t_consumed) {
    if (q.n == 0) {
        cigar->clear();
        *ed = 0;
        *t_consumed = 0;
        return true;
    }
    const int32_t qn = q.n, tn = t.n;
    if (tn <= qn + qn / 2 + 10) {
        int32_t e = 0;
        *cigar = fill_wfa(q, t, &e);
        if (max_s_cap >= 0 && e > max_s_cap) return false;
        *ed = e;
        *t_consumed = tn;
        return true;
    }
    const size_t size = static_cast<size_t>(qn + tn + 1);
    std::vector<LinFrame> hist;
    LinFrame cur{std::vector<int32_t>(size, UNSET), std::vector<uint8_t>(size, 0)};
    cur.wf[tn] = wfa_extend_diag(q, t, 0, 0);
    const int32_t max_s = qn + tn;
    int32_t explore = max_s;
    if (max_s_cap >= 0 && max_s_cap < max_s) explore = static_cast<int32_t>(max_s_cap);
    int32_t te = 0;
    if (fitting_end_k(cur.wf, qn, tn, &te)) {
        hist.push_back(std::move(cur));
        *cigar = lin_traceback(hist, q, t, 0, te);
        *ed = 0;
        *t_consumed = te;
        return true;
    }
    hist.push_back(std::move(cur));
    for (int32_t s = 1; s <= explore; ++s) {
        LinFrame next{std::vector<int32_t>(size, UNSET), std::vector<uint8_t>(size, 0)};
        lin_step(hist[s - 1], next, q, t, s);
        bool found = fitting_end_k(next.wf, qn, tn, &te);
        hist.push_back(std::move(next));
        if (found) {
            *cigar = lin_traceback(hist, q, t, s, te);
            *ed = s;
            *t_consumed = te;
            return true;
        }
    }
    return false;
}

// ---------------------------------------------------------------------------
// Gap-affine WFA, literal restatement (wfa_simd.rs:549-935).
// ---------------------------------------------------------------------------
struct AffFrame {
    std::vector<int32_t> m, ins, del;
    std::vector<uint8_t> m_op, ins_op, del_op;
};

// affine_pos_valid (wfa_simd.rs:563-569).
inline bool aff_valid(int32_t pos, int32_t k, int32_t qn, int32_t tn) {
    if (pos == UNSET || pos < 0 || pos > qn) return false;
    int32_t tp = pos - k;
    return tp >= 0 && tp <= tn;
}

// affine_traceback (wfa_simd.rs:785-886).
std::string affine_traceback(const std::vector<AffFrame>& hist, const Seq& q, const Seq& t,
                             int32_t s_end, int32_t t_end, int32_t k_end, uint8_t start_layer,
                             const phr_affine_costs& c) {
    const int32_t tn = t.n;
    std::vector<char> ops;
    int32_t qi = q.n, ti = t_end, k = k_end, s = s_end;
    uint8_t layer = start_layer;
    while (qi > 0 || ti > 0) {
        if (s == 0) {
            while (qi > 0 && ti > 0) {
                ops.push_back('M');
                --qi;
                --ti;
            }
            break;
        }
        size_t ki = static_cast<size_t>(k + tn);
        const AffFrame& f = hist[s];
        if (layer == 0) {
            uint8_t mo = f.m_op[ki];
            if (mo == 0) {
                int32_t s_mm = s - c.mismatch;
                int32_t raw = hist[s_mm].m[ki] + 1;
                for (int32_t r = 0; r < std::max(qi - raw, 0); ++r) {
                    ops.push_back('M');
                }
                int32_t n = std::max(qi - raw, 0);
                qi -= n;
                ti -= n;
                ops.push_back('X');
                --qi;
                --ti;
                s = s_mm;
            } else {
                int32_t raw = (mo == 1) ? f.ins[ki] : f.del[ki];
                int32_t n = std::max(qi - raw, 0);
                for (int32_t r = 0; r < n; ++r) ops.push_back('M');
                qi -= n;
                ti -= n;
                layer = (mo == 1) ? 1 : 2;
            }
        } else if (layer == 1) {
            ops.push_back('D');
            --qi;
            if (f.ins_op[ki] == 0) {
                s -= c.gap_open + c.gap_extend;
                k -= 1;
                layer = 0;
            } else {
                s -= c.gap_extend;
                k -= 1;
            }
        } else {
            ops.push_back('I');
            --ti;
            if (f.del_op[ki] == 0) {
                s -= c.gap_open + c.gap_extend;
                k += 1;
                layer = 0;
            } else {
                s -= c.gap_extend;
                k += 1;
            }
        }
    }
    std::reverse(ops.begin(), ops.end());
    return compact_cigar(ops);
}

// levenshtein_from_cigar (wfa_simd.rs:893-908): X count plus I/D run lengths.
int32_t levenshtein_from_cigar(const std::string& cigar) {
    int64_t total = 0, num = 0;
    for (char ch : cigar) {
        if (ch >= '0' && ch <= '9') {
            num = num * 10 + (ch - '0');
        } else {
            if (ch != 'M') total += num;
            num = 0;
        }
    }
    return static_cast<int32_t>(total);
}

// fill_wfa_affine_generic (wfa_simd.rs:581-779). Returns false when abandoned.
bool fill_wfa_affine_generic(const Seq& q, const Seq& t, const phr_affine_costs& c, bool fitting,
                             int64_t max_s_cap, std::string* cigar, int32_t* score,
                             int32_t* t_consumed) {
    const int32_t qn = q.n, tn = t.n;
    if (qn == 0 && tn == 0) {
        cigar->clear();
        *score = 0;
        *t_consumed = 0;
        return true;
    }
    if (qn == 0) {
        if (fitting) {
            cigar->clear();
            *score = 0;
            *t_consumed = 0;
        } else {
            *cigar = std::to_string(tn) + "I";
            *score = c.gap_open + tn * c.gap_extend;
            *t_consumed = tn;
        }
        return true;
    }
    const size_t size = static_cast<size_t>(qn + tn + 1);
    const int32_t diag_lo = -tn, diag_hi = qn;

    // endpoint closure (wfa_simd.rs:618-650)
    auto endpoint = [&](const AffFrame& f, int32_t* te_out, int32_t* k_out, uint8_t* layer_out) {
        auto check = [&](size_t ki, uint8_t* layer) -> bool {
            if (ki < f.m.size() && f.m[ki] == qn) { *layer = 0; return true; }
            if (ki < f.ins.size() && f.ins[ki] == qn) { *layer = 1; return true; }
            if (ki < f.del.size() && f.del[ki] == qn) { *layer = 2; return true; }
            return false;
        };
        if (!fitting) {
            int32_t k = qn - tn;
            uint8_t layer;
            if (check(static_cast<size_t>(k + tn), &layer)) {
                *te_out = tn;
                *k_out = k;
                *layer_out = layer;
                return true;
            }
            return false;
        }
        bool found = false;
        for (int32_t k = qn - tn; k <= qn; ++k) {
            int32_t te = qn - k;
            if (te < 0 || te > tn) continue;
            uint8_t layer;
            if (check(static_cast<size_t>(k + tn), &layer)) {
                if (!found || te > *te_out) {
                    *te_out = te;
                    *k_out = k;
                    *layer_out = layer;
                    found = true;
                }
            }
        }
        return found;
    };

    std::vector<AffFrame> hist;
    {
        AffFrame f0;
        f0.m.assign(size, UNSET);
        f0.ins.assign(size, UNSET);
        f0.del.assign(size, UNSET);
        f0.m_op.assign(size, 0);
        f0.ins_op.assign(size, 0);
        f0.del_op.assign(size, 0);
        f0.m[tn] = wfa_extend_diag(q, t, 0, 0);
        hist.push_back(std::move(f0));
    }
    int32_t te = 0, ke = 0;
    uint8_t layer = 0;
    if (endpoint(hist[0], &te, &ke, &layer)) {
        *cigar = affine_traceback(hist, q, t, 0, te, ke, layer, c);
        *score = 0;
        *t_consumed = te;
        return true;
    }
    const int64_t hard_max_s = static_cast<int64_t>(qn + tn) * std::max(c.mismatch, 1) + c.gap_open +
                               c.gap_extend + 4;
    int64_t explore_to = hard_max_s;
    if (max_s_cap >= 0) explore_to = std::min(max_s_cap, hard_max_s);

    for (int32_t s = 1; s <= explore_to; ++s) {
        AffFrame f;
        f.ins.assign(size, UNSET);
        f.ins_op.assign(size, 0);
        f.del.assign(size, UNSET);
        f.del_op.assign(size, 0);
        const int32_t s_open = s - c.gap_open - c.gap_extend;
        const int32_t s_ext = s - c.gap_extend;
        for (int32_t k = diag_lo; k <= diag_hi; ++k) {
            const size_t ki = static_cast<size_t>(k + tn);
            // ins (wfa_simd.rs:683-708)
            int32_t best = UNSET;
            uint8_t bop = 0;
            if (s_open >= 0 && k - 1 >= diag_lo) {
                const AffFrame& p = hist[s_open];
                size_t pk = static_cast<size_t>(k - 1 + tn);
                if (pk < p.m.size() && p.m[pk] != UNSET) {
                    int32_t cand = p.m[pk] + 1;
                    if (aff_valid(cand, k, qn, tn) && cand > best) { best = cand; bop = 0; }
                }
            }
            if (s_ext >= 0 && k - 1 >= diag_lo) {
                const AffFrame& p = hist[s_ext];
                size_t pk = static_cast<size_t>(k - 1 + tn);
                if (pk < p.ins.size() && p.ins[pk] != UNSET) {
                    int32_t cand = p.ins[pk] + 1;
                    if (aff_valid(cand, k, qn, tn) && cand > best) { best = cand; bop = 1; }
                }
            }
            if (best != UNSET) {
                f.ins[ki] = best;
                f.ins_op[ki] = bop;
            }
            // del (wfa_simd.rs:710-737)
            best = UNSET;
            bop = 0;
            if (s_open >= 0 && k + 1 <= diag_hi) {
                const AffFrame& p = hist[s_open];
                size_t pk = static_cast<size_t>(k + 1 + tn);
                if (pk < p.m.size() && p.m[pk] != UNSET) {
                    int32_t cand = p.m[pk];
                    if (aff_valid(cand, k, qn, tn) && cand > best) { best = cand; bop = 0; }
                }
            }
            if (s_ext >= 0 && k + 1 <= diag_hi) {
                const AffFrame& p = hist[s_ext];
                size_t pk = static_cast<size_t>(k + 1 + tn);
                if (pk < p.del.size() && p.del[pk] != UNSET) {
                    int32_t cand = p.del[pk];
                    if (aff_valid(cand, k, qn, tn) && cand > best) { best = cand; bop = 1; }
                }
            }
            if (best != UNSET) {
                f.del[ki] = best;
                f.del_op[ki] = bop;
            }
        }
        // m (wfa_simd.rs:740-765)
        f.m.assign(size, UNSET);
        f.m_op.assign(size, 0);
        const int32_t s_mm = s - c.mismatch;
        for (int32_t k = diag_lo; k <= diag_hi; ++k) {
            const size_t ki = static_cast<size_t>(k + tn);
            int32_t best = UNSET;
            uint8_t bop = 0;
            if (s_mm >= 0) {
                const AffFrame& p = hist[s_mm];
                if (ki < p.m.size() && p.m[ki] != UNSET) {
                    int32_t cand = p.m[ki] + 1;
                    if (aff_valid(cand, k, qn, tn) && cand > best) { best = cand; bop = 0; }
                }
            }
            if (f.ins[ki] != UNSET && aff_valid(f.ins[ki], k, qn, tn) && f.ins[ki] > best) {
                best = f.ins[ki];
                bop = 1;
            }
            if (f.del[ki] != UNSET && aff_valid(f.del[ki], k, qn, tn) && f.del[ki] > best) {
                best = f.del[ki];
                bop = 2;
            }
            if (best != UNSET) {
                f.m[ki] = wfa_extend_diag(q, t, best, k);
                f.m_op[ki] = bop;
            }
        }
        hist.push_back(std::move(f));
        if (endpoint(hist[s], &te, &ke, &layer)) {
            *cigar = affine_traceback(hist, q, t, s, te, ke, layer, c);
            *score = s;
            *t_consumed = te;
            return true;
        }
    }
    return false;
}

// fill_wfa_affine_fitting_impl (wfa_simd.rs:919-935).
bool fill_wfa_affine_fitting_impl(const Seq& q, const Seq& t, const phr_affine_costs& c,
                                  int64_t max_s_cap, std::string* cigar, int32_t* ed,
                                  int32_t* t_end, int32_t* score) {
    if (q.n == 0) {
        cigar->clear();
        *ed = 0;
        *t_end = 0;
        *score = 0;
        return true;
    }
    const int32_t qn = q.n, tn = t.n;
    const bool fitting = tn > qn + qn / 2 + 10;
    if (!fill_wfa_affine_generic(q, t, c, fitting, max_s_cap, cigar, score, t_end)) return false;
    *ed = levenshtein_from_cigar(*cigar);
    return true;
}

// ---------------------------------------------------------------------------
// Myers bit-parallel, literal restatement (wfa_simd.rs:3507-3814).
// ---------------------------------------------------------------------------
struct MyersColumns {
    std::vector<uint64_t> data;
    std::vector<int64_t> scores;
    size_t num_blocks = 0;
    size_t num_cols = 0;
};

// myers_forward_flat_with_cutoff (wfa_simd.rs:3552-3648). margin < 0: no cutoff.
MyersColumns myers_forward(const Seq& query, const Seq& target, int64_t margin) {
    constexpr size_t W = 64;
    const size_t m = static_cast<size_t>(query.n), n = static_cast<size_t>(target.n);
    const size_t nb = (m + W - 1) / W;
    const size_t last_block = nb - 1;
    const size_t last_bits = (m % W == 0) ? W : m % W;
    const uint64_t last_mask = (last_bits == W) ? ~0ull : ((1ull << last_bits) - 1);
    const size_t score_bit = (m - 1) % W;
    std::vector<uint64_t> pm(nb * 256, 0);
    for (size_t i = 0; i < m; ++i) pm[(i / W) * 256 + query.p[i]] |= 1ull << (i % W);
    std::vector<uint64_t> vp(nb, ~0ull), vn(nb, 0), nvp(nb), nvn(nb);
    vp[last_block] = last_mask;
    int64_t score = static_cast<int64_t>(m), best_seen = static_cast<int64_t>(m);
    const size_t stride = nb * 2;
    MyersColumns out;
    out.num_blocks = nb;
    out.data.assign(n * stride, 0);
    out.scores.reserve(n);
    for (size_t col = 0; col < n; ++col) {
        const uint8_t tb = target.p[col];
        uint64_t add_carry = 0, hp_carry = 1, hn_carry = 0, last_hp = 0, last_hn = 0;
        for (size_t k = 0; k < nb; ++k) {
            uint64_t eq = pm[k * 256 + tb];
            uint64_t xh = eq | vn[k];
            uint64_t xhvp = xh & vp[k];
            uint64_t s1 = vp[k] + xhvp;
            uint64_t c1 = s1 < vp[k] ? 1 : 0;
            uint64_t s2 = s1 + add_carry;
            uint64_t c2 = s2 < s1 ? 1 : 0;
            add_carry = c1 | c2;
            uint64_t d0 = (s2 ^ vp[k]) | xh;
            uint64_t hn = vp[k] & d0;
            uint64_t hp = vn[k] | ~(vp[k] | d0);
            const bool partial = (k == last_block && last_bits < W);
            if (partial) {
                d0 &= last_mask;
                hn &= last_mask;
                hp &= last_mask;
            }
            if (k == last_block) {
                last_hp = hp;
                last_hn = hn;
            }
            uint64_t nhp = hp >> (W - 1);
            uint64_t x = (hp << 1) | hp_carry;
            hp_carry = nhp;
            uint64_t nhn = hn >> (W - 1);
            uint64_t hns = (hn << 1) | hn_carry;
            hn_carry = nhn;
            nvn[k] = x & d0;
            uint64_t v2 = hns | ~(d0 | x);
            nvp[k] = partial ? (v2 & last_mask) : v2;
        }
        if ((last_hp >> score_bit) & 1) score += 1;
        if ((last_hn >> score_bit) & 1) score = score > 0 ? score - 1 : 0;
        std::swap(vp, nvp);
        std::swap(vn, nvn);
        std::memcpy(&out.data[col * stride], vp.data(), nb * 8);
        std::memcpy(&out.data[col * stride + nb], vn.data(), nb * 8);
        out.scores.push_back(score);
        if (score < best_seen) best_seen = score;
        if (margin >= 0 && score > best_seen + margin) {
            out.num_cols = col + 1;
            out.data.resize(out.num_cols * stride);
            return out;
        }
    }
    out.num_cols = n;
    return out;
}

// fill_dp_column_flat (wfa_simd.rs:3689-3699) + reconstruct_into (:3507-3516).
void fill_col(const MyersColumns& cols, size_t m, size_t j, std::vector<int64_t>& buf) {
    if (j == 0) {
        for (size_t i = 0; i <= m; ++i) buf[i] = static_cast<int64_t>(i);
        return;
    }
    const size_t nb = cols.num_blocks;
    const uint64_t* vp = &cols.data[(j - 1) * nb * 2];
    const uint64_t* vn = vp + nb;
    buf[m] = cols.scores[j - 1];
    for (size_t i = m; i-- > 0;) {
        int64_t vpb = static_cast<int64_t>((vp[i / 64] >> (i % 64)) & 1);
        int64_t vnb = static_cast<int64_t>((vn[i / 64] >> (i % 64)) & 1);
        buf[i] = buf[i + 1] - vpb + vnb;
    }
}

// myers_backtrace_flat (wfa_simd.rs:3702-3781). Precedence D (above), I (left), diagonal.
std::string myers_backtrace(const Seq& query, const Seq& target, const MyersColumns& cols,
                            size_t end_ti) {
    const size_t m = static_cast<size_t>(query.n);
    std::vector<char> ops;
    ops.reserve(m + end_ti);
    size_t qi = m, ti = end_ti;
    std::vector<int64_t> cur(m + 1, 0), prev(m + 1, 0);
    if (ti > 0) {
        fill_col(cols, m, ti, cur);
        fill_col(cols, m, ti - 1, prev);
    }
    while (qi > 0 || ti > 0) {
        if (qi == 0) {
            ops.push_back('I');
            --ti;
            continue;
        }
        if (ti == 0) {
            ops.push_back('D');
            --qi;
            continue;
        }
        int64_t c = cur[qi];
        int64_t diag_cost = query.p[qi - 1] == target.p[ti - 1] ? 0 : 1;
        int64_t from_above = cur[qi - 1] + 1;
        int64_t from_left = prev[qi] + 1;
        if (c == from_above) {
            ops.push_back('D');
            --qi;
        } else if (c == from_left) {
            ops.push_back('I');
            --ti;
            std::swap(cur, prev);
            if (ti > 0) fill_col(cols, m, ti - 1, prev);
        } else {
            ops.push_back(diag_cost == 0 ? 'M' : 'X');
            --qi;
            --ti;
            std::swap(cur, prev);
            if (ti > 0) fill_col(cols, m, ti - 1, prev);
        }
    }
    std::reverse(ops.begin(), ops.end());
    return compact_cigar(ops);
}

// myers_edit_distance_impl (wfa_simd.rs:3657-3673).
void myers_global(const Seq& q, const Seq& t, int32_t* ed, std::string* cigar) {
    if (q.n == 0) {
        *cigar = t.n > 0 ? std::to_string(t.n) + "I" : std::string();
        *ed = t.n;
        return;
    }
    if (t.n == 0) {
        *cigar = std::to_string(q.n) + "D";
        *ed = q.n;
        return;
    }
    MyersColumns cols = myers_forward(q, t, -1);
    *ed = cols.num_cols > 0 ? static_cast<int32_t>(cols.scores[cols.num_cols - 1]) : q.n;
    *cigar = myers_backtrace(q, t, cols, static_cast<size_t>(t.n));
}

// myers_fitting_impl (wfa_simd.rs:3783-3814).
void myers_fitting(const Seq& q, const Seq& t, int32_t* ed, std::string* cigar, int32_t* consumed) {
    const int32_t m = q.n, n = t.n;
    if (m == 0) {
        *ed = 0;
        cigar->clear();
        *consumed = 0;
        return;
    }
    if (n == 0) {
        *ed = m;
        *cigar = std::to_string(m) + "D";
        *consumed = 0;
        return;
    }
    if (n <= m + m / 2 + 10) {
        myers_global(q, t, ed, cigar);
        *consumed = n;
        return;
    }
    const int64_t margin = m / 10 + 1;
    MyersColumns cols = myers_forward(q, t, margin);
    size_t best_consumed = 0;
    int64_t best_score = m;
    for (size_t c = 0; c < cols.num_cols; ++c) {
        if (cols.scores[c] < best_score) {
            best_score = cols.scores[c];
            best_consumed = c + 1;
        }
    }
    *cigar = myers_backtrace(q, t, cols, best_consumed);
    *ed = static_cast<int32_t>(best_score);
    *consumed = static_cast<int32_t>(best_consumed);
}

// ---------------------------------------------------------------------------
// Public alignment entry points (phraya-align/src/lib.rs:63-167).
// ---------------------------------------------------------------------------
struct Aln {
    int32_t status = PHR_OK;
    std::string cigar;
    int32_t ed = 0;
    int32_t qs = 0, qe = 0, ts = 0, te = 0;
    int32_t affine_score = 0;
    bool operator==(const Aln& o) const {
        return cigar == o.cigar && ed == o.ed && qs == o.qs && qe == o.qe && ts == o.ts && te == o.te;
    }
};

Aln extend_one(phr_engine engine, const uint8_t* q, int32_t qlen, const uint8_t* t, int32_t tlen,
               int32_t qseed, int32_t tseed, const phr_affine_costs& costs) {
    Aln a;
    if (engine == PHR_ENGINE_MYERS_GLOBAL) {
        // myers_edit_distance (lib.rs:94-96): whole sequences, no anchor.
        Seq qs{q, qlen}, ts{t, tlen};
        myers_global(qs, ts, &a.ed, &a.cigar);
        a.qs = 0;
        a.qe = qlen;
        a.ts = 0;
        a.te = tlen;
        return a;
    }
    // lib.rs:107-111 / :145-149 / wfa_simd.rs:175-179: seed beyond the end.
    if (qseed > qlen || tseed > tlen) {
        a.status = PHR_INVALID_INPUT;
        return a;
    }
    Seq qs{q + qseed, qlen - qseed}, ts{t + tseed, tlen - tseed};
    a.qs = qseed;
    a.qe = qseed + qs.n;
    a.ts = tseed;
    if (engine == PHR_ENGINE_MYERS_FIT) {
        int32_t cons = 0;
        myers_fitting(qs, ts, &a.ed, &a.cigar, &cons);
        a.te = tseed + cons;
        return a;
    }
    if (engine == PHR_ENGINE_WFA_LINEAR) {
        // wfa_extend_naive_impl (wfa_simd.rs:173-223)
        if (qs.n == 0 && ts.n == 0) {
            a.te = tseed;
            return a;
        }
        int32_t cons = 0;
        if (!fill_wfa_fitting_impl(qs, ts, -1, &a.cigar, &a.ed, &cons)) {
            a.status = PHR_ALIGNMENT_FAILED;
            a.cigar.clear();
            return a;
        }
        a.te = tseed + cons;
        return a;
    }
    // PHR_ENGINE_WFA_AFFINE: wfa_extend_affine (lib.rs:139-167)
    int32_t te = 0, score = 0;
    if (!fill_wfa_affine_fitting_impl(qs, ts, costs, -1, &a.cigar, &a.ed, &te, &score)) {
        a.status = PHR_ALIGNMENT_FAILED;
        a.cigar.clear();
        return a;
    }
    a.te = tseed + te;
    a.affine_score = score;
    return a;
}

// ---------------------------------------------------------------------------
// Minimizer sketcher: simd-minimizers' random minimizers restated from their published
// descriptions (the crate is not in the reference tree).
//   * Characters: packed-seq's AsciiSeq view, which the call site uses for DNA and
//     protein alike (types.rs:1849-1862): 2 bits per character, code(b) = (b >> 1) & 3,
//     i.e. A = 0, C = 1, T = 2, G = 3 for either case; the complement is code ^ 2.
//   * Order hash: ntHash (Mohamadi et al., Bioinformatics 2016; "ntHash rolling hashes",
//     README.md:185) in 32 bits, the lane width of the SIMD sketcher (Groot Koerkamp &
//     Martayan, SEA 2025): h_fw = XOR_i rotl(seed[x_i], k-1-i), h_rc = XOR_i
//     rotl(seed[comp(x_i)], i), over the four published ntHash base seeds (low 32 bits).
//     Canonical (DNA): min(h_fw, h_rc), ntHash's canonical hash; plain (protein): h_fw.
//   * Window: w consecutive k-mers (l = w + k - 1 characters). Plain minimizers take the
//     leftmost minimum hash. Canonical minimizers (odd l, README.md:190) orient each
//     window by its characters: a window with more T/G than A/C (codes 2, 3 against
//     0, 1) is forward and takes the leftmost minimum, otherwise the rightmost, so a
//     sequence and its reverse complement select the same k-mers (SEA 2025).
//   * Output: each selected k-mer once per run of windows selecting it (the crate's
//     minimizer positions), paired with its value (`pos_and_values_u64`): the 2-bit
//     k-mer, first character in the low bits; canonical: min(forward, reverse
//     complement) (docs/adr/0013-protein-space-alphabet-support.md:20-21).
// ---------------------------------------------------------------------------
constexpr uint32_t kNtSeed[4] = {
    static_cast<uint32_t>(0x3c8bfbb395c60474ull),  // A (code 0)
    static_cast<uint32_t>(0x3193c18562a02b4cull),  // C (code 1)
    static_cast<uint32_t>(0x295549f54be24456ull),  // T (code 2)
    static_cast<uint32_t>(0x20323ed082572324ull),  // G (code 3)
};

inline uint32_t rotl32(uint32_t x, int r) {
    r &= 31;
    return r ? (x << r) | (x >> (32 - r)) : x;
}

void sketch_seq(const uint8_t* s, int64_t len, int k, int w, int alphabet,
                std::vector<std::pair<uint64_t, uint32_t>>* out) {
    out->clear();
    if (k <= 0 || w <= 0 || k > 32 || len < k) return;
    const bool canonical = alphabet == PHR_ALPHABET_DNA;
    const int64_t nk = len - k + 1;
    std::vector<uint32_t> hash(static_cast<size_t>(nk));
    std::vector<uint64_t> value(static_cast<size_t>(nk));
    for (int64_t p = 0; p < nk; ++p) {
        uint32_t hf = 0, hr = 0;
        uint64_t vf = 0, vr = 0;
        for (int i = 0; i < k; ++i) {
            const uint32_t c = (s[p + i] >> 1) & 3;
            hf ^= rotl32(kNtSeed[c], k - 1 - i);
            hr ^= rotl32(kNtSeed[c ^ 2], i);
            vf |= static_cast<uint64_t>(c) << (2 * i);
            vr |= static_cast<uint64_t>(c ^ 2) << (2 * (k - 1 - i));
        }
        hash[static_cast<size_t>(p)] = canonical ? std::min(hf, hr) : hf;
        value[static_cast<size_t>(p)] = canonical ? std::min(vf, vr) : vf;
    }
    if (nk < w) return;
    const int64_t l = w + k - 1;
    int64_t last = -1;
    for (int64_t ws = 0; ws + w <= nk; ++ws) {
        bool forward = true;
        if (canonical) {
            int64_t tg = 0;
            for (int64_t i = ws; i < ws + l; ++i) tg += ((s[i] >> 1) & 2) ? 1 : 0;
            forward = 2 * tg > l;
        }
        int64_t best = ws;
        for (int64_t p = ws + 1; p < ws + w; ++p) {
            const uint32_t a = hash[static_cast<size_t>(p)], b = hash[static_cast<size_t>(best)];
            if (a < b || (!forward && a == b)) best = p;
        }
        if (best != last) {
            out->push_back({value[static_cast<size_t>(best)], static_cast<uint32_t>(best)});
            last = best;
        }
    }
}

// ---------------------------------------------------------------------------
// Seeding (phraya-align/src/seeding.rs:31-102) and chaining (chaining.rs:96-226).
// ---------------------------------------------------------------------------
struct SeedT {
    uint32_t qpos, tpos;
    uint64_t val;
};

struct Index {
    std::unordered_map<uint64_t, std::vector<uint32_t>> map;
    uint64_t cap = 256;
};

// build_minimizer_index (seeding.rs:31-37) + seed_occurrence_cap (:94-102).
void build_index(const std::vector<std::pair<uint64_t, uint32_t>>& sk, uint64_t floor, Index* idx) {
    idx->map.clear();
    for (auto& e : sk) idx->map[e.first].push_back(e.second);
    if (idx->map.empty()) {
        idx->cap = floor;
        return;
    }
    std::vector<uint64_t> counts;
    counts.reserve(idx->map.size());
    for (auto& kv : idx->map) counts.push_back(kv.second.size());
    std::sort(counts.begin(), counts.end());
    uint64_t median = counts[counts.size() / 2];
    idx->cap = std::max<uint64_t>(floor, median * 8);
}

// find_seeds_indexed_capped (seeding.rs:58-80): emit in query-sketch order, then a
// stable sort by query_pos.
std::vector<SeedT> find_seeds(const std::vector<std::pair<uint64_t, uint32_t>>& qsk, const Index& idx) {
    std::vector<SeedT> seeds;
    for (auto& e : qsk) {
        auto it = idx.map.find(e.first);
        if (it == idx.map.end()) continue;
        if (it->second.size() > idx.cap) continue;
        for (uint32_t tp : it->second) seeds.push_back({e.second, tp, e.first});
    }
    std::stable_sort(seeds.begin(), seeds.end(),
                     [](const SeedT& a, const SeedT& b) { return a.qpos < b.qpos; });
    return seeds;
}

struct ChainT {
    std::vector<SeedT> seeds;
    int64_t score;
    uint32_t target_start() const {  // Chain::target_start (chaining.rs:32-35)
        int64_t v = static_cast<int64_t>(seeds[0].tpos) - static_cast<int64_t>(seeds[0].qpos);
        return static_cast<uint32_t>(v > 0 ? v : 0);
    }
};

struct ChainParams {  // ChainParams::default (chaining.rs:75-86)
    int64_t seed_len = 21, max_band = 100, max_dist_x = 100;
    size_t max_iter = 5000, max_skip = 25;
    double gap_penalty = 0.21;
    int64_t min_chain_score = 25;
};

// chain_score (chaining.rs:96-117). Returns false for "None".
bool chain_score(const SeedT& si, const SeedT& sj, const ChainParams& p, int64_t* sc_out) {
    int64_t dq = static_cast<int64_t>(si.qpos) - static_cast<int64_t>(sj.qpos);
    if (dq <= 0) return false;
    int64_t dr = static_cast<int64_t>(si.tpos) - static_cast<int64_t>(sj.tpos);
    if (dr <= 0 || dr > p.max_dist_x + p.seed_len) return false;
    int64_t dd = dr > dq ? dr - dq : dq - dr;
    if (dd > p.max_band) return false;
    int64_t dg = std::min(dr, dq);
    int64_t sc = std::min(p.seed_len, dg);
    if (dd > 0) {
        double lin = p.gap_penalty * static_cast<double>(dd);
        double lg = 0.5 * std::log2(static_cast<double>(dd) + 1.0);
        sc -= static_cast<int64_t>(std::round(lin + lg));  // Rust f64::round: half away from 0
    }
    *sc_out = sc;
    return true;
}

// chain_seeds (chaining.rs:134-226).
std::vector<ChainT> chain_seeds(const std::vector<SeedT>& seeds, const ChainParams& p) {
    std::vector<ChainT> chains;
    if (seeds.empty()) return chains;
    std::vector<SeedT> sorted = seeds;
    std::stable_sort(sorted.begin(), sorted.end(), [](const SeedT& a, const SeedT& b) {
        return a.tpos != b.tpos ? a.tpos < b.tpos : a.qpos < b.qpos;
    });
    const size_t n = sorted.size();
    std::vector<int64_t> f(n, 0);
    std::vector<int64_t> pred(n, -1);
    std::vector<size_t> dominated(n, 0);
    for (size_t i = 0; i < n; ++i) {
        int64_t best_score = p.seed_len;
        int64_t best_pred = -1;
        size_t n_skip = 0;
        size_t floor = i > p.max_iter ? i - p.max_iter : 0;
        for (size_t j = i; j-- > floor;) {
            if (static_cast<int64_t>(sorted[i].tpos) - static_cast<int64_t>(sorted[j].tpos) >=
                p.max_dist_x + p.seed_len)
                break;
            int64_t sc;
            if (!chain_score(sorted[i], sorted[j], p, &sc)) continue;
            int64_t total = sc + f[j];
            if (total > best_score) {
                best_score = total;
                best_pred = static_cast<int64_t>(j);
                if (n_skip > 0) --n_skip;
            } else {
                dominated[j] += 1;
                if (dominated[j] > p.max_skip) {
                    n_skip += 1;
                    if (n_skip > p.max_skip) break;
                }
            }
        }
        f[i] = best_score;
        pred[i] = best_pred;
    }
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return f[a] > f[b]; });
    std::vector<bool> used(n, false);
    for (size_t end : order) {
        if (used[end] || f[end] < p.min_chain_score) continue;
        std::vector<SeedT> rev;
        int64_t cur = static_cast<int64_t>(end);
        while (cur >= 0) {
            if (used[cur]) break;
            used[cur] = true;
            rev.push_back(sorted[cur]);
            cur = pred[cur];
        }
        if (rev.empty()) continue;
        std::reverse(rev.begin(), rev.end());
        std::stable_sort(rev.begin(), rev.end(),
                         [](const SeedT& a, const SeedT& b) { return a.qpos < b.qpos; });
        chains.push_back({std::move(rev), f[end]});
    }
    std::stable_sort(chains.begin(), chains.end(),
                     [](const ChainT& a, const ChainT& b) { return a.score > b.score; });
    return chains;
}

// ---------------------------------------------------------------------------
// align_read (phraya-align/src/executor.rs:573-733), up to the scored alignments.
// ---------------------------------------------------------------------------
struct Scored {
    Aln primary;
    std::vector<Aln> alts;
};

// score_alignments (lib.rs:170-199).
Scored score_alignments(const std::vector<Aln>& alns, size_t query_len) {
    Scored s;
    size_t pi = 0;
    for (size_t i = 1; i < alns.size(); ++i)
        if (alns[i].ed < alns[pi].ed) pi = i;  // min_by_key keeps the FIRST minimum
    s.primary = alns[pi];
    const double ql = static_cast<double>(query_len);
    for (const Aln& a : alns) {
        if (a == s.primary) continue;
        double pn = 1.0 - (static_cast<double>(s.primary.ed) / ql);
        double an = 1.0 - (static_cast<double>(a.ed) / ql);
        if (an / pn >= 0.95) s.alts.push_back(a);
    }
    return s;
}

// reverse_complement (phraya-core/src/types.rs:91-107).
std::vector<uint8_t> revcomp(const uint8_t* s, size_t n) {
    std::vector<uint8_t> out(n);
    for (size_t i = 0; i < n; ++i) {
        uint8_t b = s[n - 1 - i];
        switch (b) {
            case 'A': b = 'T'; break;
            case 'T': b = 'A'; break;
            case 'C': b = 'G'; break;
            case 'G': b = 'C'; break;
            case 'a': b = 't'; break;
            case 't': b = 'a'; break;
            case 'c': b = 'g'; break;
            case 'g': b = 'c'; break;
            default: break;
        }
        out[i] = b;
    }
    return out;
}

// RepeatRegion (phraya-core/src/lib.rs:10-18) without its period/unit strings.
struct RepeatRegionT {
    size_t start, end;  // end inclusive
};

std::vector<RepeatRegionT> detect_tandem_repeats(const uint8_t* seq, size_t n, size_t min_count);

struct Target {
    std::vector<uint8_t> bytes;
    Index index;
    int alphabet = PHR_ALPHABET_DNA;
    std::vector<RepeatRegionT> repeats;  // TargetContext::repeat_regions (executor.rs:440-441)
};

size_t chain_cap(int strategy) { return strategy == PHR_FAST ? 1 : strategy == PHR_BALANCED ? 2 : 50; }

// anchors_from_chains (executor.rs:347-362): the target starts of the first K chains
// (K = chain_cap), or the origin when there is no chain. Only target positions vary (the
// query position of every anchor is 0).
std::vector<uint32_t> anchors_from_chains(const std::vector<uint32_t>& chain_starts, int strategy) {
    std::vector<uint32_t> anchors;
    if (chain_starts.empty()) {
        anchors.push_back(0);
    } else {
        const size_t K = std::min(chain_cap(strategy), chain_starts.size());
        for (size_t i = 0; i < K; ++i) anchors.push_back(chain_starts[i]);
    }
    return anchors;
}

// extend_chains (executor.rs:528-567) with anchors_from_chains and extend_anchor
// (:379-404). Returns false for None.
bool extend_chains(const Target& tg, const phr_align_config& cfg, const uint8_t* q, size_t qlen,
                   const std::vector<ChainT>& chains, Scored* out) {
    std::vector<uint32_t> starts;
    for (const ChainT& c : chains) starts.push_back(c.target_start());
    const std::vector<uint32_t> anchors = anchors_from_chains(starts, cfg.strategy);
    std::vector<Aln> alns;
    const phr_affine_costs def_costs{2, 4, 1};
    for (uint32_t a : anchors) {
        size_t wend = std::min<size_t>(static_cast<size_t>(a) + qlen * 2, tg.bytes.size());
        phr_engine eng;
        if (cfg.strategy == PHR_SENSITIVE)
            eng = cfg.gap_model == PHR_GAP_AFFINE ? PHR_ENGINE_WFA_AFFINE : PHR_ENGINE_WFA_LINEAR;
        else
            eng = qlen <= 500 ? PHR_ENGINE_MYERS_FIT : PHR_ENGINE_WFA_LINEAR;
        Aln r = extend_one(eng, q, static_cast<int32_t>(qlen), tg.bytes.data(),
                           static_cast<int32_t>(wend), 0, static_cast<int32_t>(a), def_costs);
        if (r.status == PHR_OK) alns.push_back(std::move(r));
    }
    if (alns.empty()) return false;
    *out = score_alignments(alns, qlen);
    return true;
}

struct ReadOut {
    int outcome = PHR_OUT_NO_ALIGNMENT;
    bool has_result = false;
    bool reverse = false;
    Scored scored;
};

void align_read(const Target& tg, const uint8_t* read, size_t len, const phr_align_config& cfg,
                const std::vector<std::pair<uint64_t, uint32_t>>* stored_fwd, ReadOut* out) {
    const bool is_dna = tg.alphabet == PHR_ALPHABET_DNA;
    const int k = is_dna ? 21 : 6, w = is_dna ? 11 : 5;
    std::vector<std::pair<uint64_t, uint32_t>> fwd_sk, rev_sk;
    bool used_stored = false;
    if (stored_fwd) {
        fwd_sk = *stored_fwd;
        used_stored = true;
    } else {
        sketch_seq(read, static_cast<int64_t>(len), k, w, tg.alphabet, &fwd_sk);
    }
    std::vector<SeedT> fseeds = find_seeds(fwd_sk, tg.index);
    ChainParams cp;
    std::vector<ChainT> fchains = chain_seeds(fseeds, cp);
    std::vector<uint8_t> rc;
    if (is_dna) rc = revcomp(read, len);
    size_t rev_seeds = 0;
    std::vector<ChainT> rchains;
    if (is_dna && !(fseeds.empty() && fwd_sk.empty())) {
        sketch_seq(rc.data(), static_cast<int64_t>(len), 21, 11, PHR_ALPHABET_DNA, &rev_sk);
        std::vector<SeedT> rseeds = find_seeds(rev_sk, tg.index);
        rev_seeds = rseeds.size();
        rchains = chain_seeds(rseeds, cp);
    }
    const bool had_seeds = !fseeds.empty() || rev_seeds > 0;
    if (used_stored && fwd_sk.empty() && !had_seeds) {
        out->outcome = PHR_OUT_NO_SEED;
        out->has_result = false;
        return;
    }
    Scored fsc, rsc;
    bool fok = false, rok = false;
    if (!fchains.empty() && rchains.empty()) {
        fok = extend_chains(tg, cfg, read, len, fchains, &fsc);
    } else if (fchains.empty() && !rchains.empty()) {
        rok = extend_chains(tg, cfg, rc.data(), rc.size(), rchains, &rsc);
    } else {
        // protein has no reverse strand: rc stays empty and is still "extended"
        // (executor.rs:633-637, 693-697)
        fok = extend_chains(tg, cfg, read, len, fchains, &fsc);
        rok = extend_chains(tg, cfg, rc.data(), rc.size(), rchains, &rsc);
    }
    if (fok && rok && rsc.primary.ed < fsc.primary.ed) {
        out->scored = std::move(rsc);
        out->reverse = true;
    } else if (fok) {
        out->scored = std::move(fsc);
        out->reverse = false;
    } else if (rok) {
        out->scored = std::move(rsc);
        out->reverse = true;
    } else {
        out->outcome = PHR_OUT_NO_ALIGNMENT;
        out->has_result = false;
        return;
    }
    const double qlen = static_cast<double>(std::max<size_t>(len, 1));
    const double primary_score = 1.0 - static_cast<double>(out->scored.primary.ed) / qlen;
    if (cfg.strategy == PHR_FAST) {
        double div = static_cast<double>(out->scored.primary.ed) / qlen;
        if (div > 0.20) {
            out->outcome = PHR_OUT_FAST_CUTOFF;
            out->has_result = false;
            out->reverse = false;  // no result: orientation is not reported
            return;
        }
    }
    out->outcome = primary_score >= 0.95 ? PHR_OUT_PLACED : (had_seeds ? PHR_OUT_BELOW_THRESHOLD : PHR_OUT_NO_SEED);
    out->has_result = true;
}

void fill_alignment(const Aln& a, phr_alignment* o, uint64_t off) {
    o->status = a.status;
    o->edit_distance = static_cast<uint32_t>(a.ed);
    o->query_start = static_cast<uint32_t>(a.qs);
    o->query_end = static_cast<uint32_t>(a.qe);
    o->target_start = static_cast<uint32_t>(a.ts);
    o->target_end = static_cast<uint32_t>(a.te);
    o->cigar_off = off;
    o->cigar_len = static_cast<uint32_t>(a.cigar.size());
    o->affine_score = static_cast<uint32_t>(a.affine_score);
}

template <class F>
void parallel_for(uint64_t n, int nthreads, F&& fn) {
    if (nthreads <= 1 || n < 2) {
        for (uint64_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<uint64_t> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t)
        th.emplace_back([&]() {
            for (;;) {
                uint64_t i = next.fetch_add(1);
                if (i >= n) break;
                fn(i);
            }
        });
    for (auto& x : th) x.join();
}

// ---------------------------------------------------------------------------
// Tandem repeats and variant observations
//   detect_tandem_repeats        phraya-core/src/lib.rs:79-135 (RepeatDetectorConfig
//                                default min_repeat_count 3, lib.rs:40-52)
//   is_in_repeat_region          phraya-align/src/executor.rs:806-809
//   is_in_hotspot                executor.rs:795-798
//   compute_windowed_coverage    executor.rs:1071-1090, WindowedCoverage::get_abs :190-197,
//                                get_abs_multi :218-220
//   extract_variants_from_cigar  executor.rs:814-1046, parse_cigar :1048-1061
//   call site / confidence       executor.rs:735-775 (primary_score = 1 - ed / max(|q|, 1))
// ---------------------------------------------------------------------------
std::vector<RepeatRegionT> detect_tandem_repeats(const uint8_t* seq, size_t n, size_t min_count) {
    std::vector<uint8_t> up(seq, seq + n);  // sequence.to_uppercase() (ASCII)
    for (uint8_t& c : up)
        if (c >= 'a' && c <= 'z') c = static_cast<uint8_t>(c - 32);
    std::vector<RepeatRegionT> regions;
    if (n < min_count * 2) return regions;
    size_t cur = 0;
    while (cur + min_count * 2 <= n) {
        bool found = false;
        for (size_t period = 4; period >= 2; --period) {  // (2..=4).rev()
            if (cur + period * min_count > n) continue;
            size_t count = 1, end = cur + period;
            while (end + period <= n && std::memcmp(&up[cur], &up[end], period) == 0) {
                ++count;
                end += period;
            }
            if (count >= min_count) {
                regions.push_back({cur, end - 1});
                cur = end;
                found = true;
                break;
            }
        }
        if (!found) ++cur;
    }
    return regions;
}

// Last region whose start <= pos; inside when pos < its (inclusive) end, as the reference.
bool in_repeat_region(size_t pos, const std::vector<RepeatRegionT>& r) {
    size_t lo = 0, hi = r.size();
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (r[mid].start <= pos) lo = mid + 1;
        else hi = mid;
    }
    return lo > 0 && pos < r[lo - 1].end;
}

bool in_hotspot(uint32_t pos, const uint32_t* hs, const uint32_t* he, size_t n) {
    size_t lo = 0, hi = n;
    while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (hs[mid] <= pos) lo = mid + 1;
        else hi = mid;
    }
    return lo > 0 && pos < he[lo - 1];
}

struct VariantOut {
    std::vector<phr_variant> v;
    std::vector<uint32_t> cov;
    std::vector<phr_allele> al;
};

// extract_variants_from_cigar for one read; windows = the read's coverage windows.
void extract_variants(const std::string& cigar, size_t target_start, const uint8_t* query, size_t qlen,
                      const uint8_t* target, size_t tlen, uint32_t ed,
                      const std::vector<std::pair<size_t, size_t>>& windows,
                      const std::vector<RepeatRegionT>& reps, const uint32_t* hs, const uint32_t* he, size_t nhs,
                      double primary_score, size_t radius, uint8_t strand, uint32_t read, VariantOut* out) {
    auto cov_at = [&](size_t pos) {  // get_abs_multi
        uint32_t c = 0;
        for (auto& w : windows)
            if (pos >= w.first && pos < w.second) c += 1;
        return c;
    };
    auto emit = [&](size_t tp, uint8_t ref, uint8_t type, const std::vector<std::pair<uint8_t, uint32_t>>& alleles) {
        phr_variant o;
        std::memset(&o, 0, sizeof(o));
        const size_t ws = tp >= radius ? tp - radius : 0;
        const size_t we = std::min(tp + radius + 1, tlen);
        o.coverage_off = out->cov.size();
        for (size_t p = ws; p < we; ++p) out->cov.push_back(cov_at(p));
        o.coverage_len = static_cast<uint32_t>(we > ws ? we - ws : 0);
        o.coverage_variant_offset = static_cast<uint32_t>(tp - ws);
        o.position = static_cast<uint32_t>(tp);
        o.ref_base = ref;
        o.variant_type = type;
        o.in_tandem_repeat = in_repeat_region(tp, reps) ? 1 : 0;
        o.strand = strand;
        o.read = read;
        o.edit_distance = ed;
        o.kmer_uniqueness = in_hotspot(static_cast<uint32_t>(tp), hs, he, nhs) ? 0.0 : 1.0;
        o.confidence = o.kmer_uniqueness * primary_score;
        o.allele_off = out->al.size();
        for (auto& a : alleles) {
            phr_allele x;
            std::memset(&x, 0, sizeof(x));
            x.base = a.first;
            x.count = a.second;
            out->al.push_back(x);
        }
        o.n_alleles = static_cast<uint32_t>(alleles.size());
        out->v.push_back(o);
    };
    size_t q = 0, t = target_start;
    size_t i = 0;
    while (i < cigar.size()) {
        size_t count = 0;
        bool digits = false;
        while (i < cigar.size() && cigar[i] >= '0' && cigar[i] <= '9') {
            count = count * 10 + static_cast<size_t>(cigar[i] - '0');
            ++i;
            digits = true;
        }
        if (i >= cigar.size()) break;
        const char op = cigar[i++];
        if (!digits) count = 1;  // count_str.parse().unwrap_or(1)
        if (op == 'M') {
            q += count;
            t += count;
        } else if (op == 'X') {
            for (size_t k = 0; k < count; ++k) {
                const size_t qp = q + k, tp = t + k;
                if (qp < qlen && tp < tlen) emit(tp, target[tp], 0, {{query[qp], 1u}});
            }
            q += count;
            t += count;
        } else if (op == 'I') {  // target-extra: deletion, ref = first deleted base, allele '.'
            if (t < tlen && q < qlen) emit(t, target[t], 2, {{static_cast<uint8_t>('.'), 1u}});
            t += count;
        } else if (op == 'D') {  // query-extra: insertion at t, alleles = inserted bases
            if (q < qlen && t < tlen) {
                std::map<uint8_t, uint32_t> m;
                for (size_t k = q; k < std::min(q + count, qlen); ++k) m[query[k]] += 1;
                std::vector<std::pair<uint8_t, uint32_t>> al(m.begin(), m.end());
                emit(t, static_cast<uint8_t>('.'), 1, al);
            }
            q += count;
        }
    }
}

}  // namespace

// ===========================================================================
// C API of the oracle (ctypes-friendly; test infrastructure only).
// ===========================================================================
extern "C" {

uint64_t orc_lcp(const uint8_t* a, uint64_t an, const uint8_t* b, uint64_t bn) { return lcp(a, an, b, bn); }

// Extends every pair of `batch` with `engine`; CIGARs are packed into out->cigar.
// Returns 0, or PHR_ERR_CAPACITY if the CIGAR arena is too small.
int32_t orc_extend_batch(int32_t engine, const phr_pair_batch* batch, phr_affine_costs costs,
                         phr_result_arena* out, int32_t nthreads) {
    const uint64_t n = batch->n_pairs;
    std::vector<Aln> res(n);
    parallel_for(n, nthreads, [&](uint64_t i) {
        const uint8_t* q = batch->seq + batch->q_off[i];
        const uint8_t* t = batch->seq + batch->t_off[i];
        int32_t qs = batch->q_seed ? static_cast<int32_t>(batch->q_seed[i]) : 0;
        int32_t ts = batch->t_seed ? static_cast<int32_t>(batch->t_seed[i]) : 0;
        res[i] = extend_one(static_cast<phr_engine>(engine), q, static_cast<int32_t>(batch->q_len[i]), t,
                            static_cast<int32_t>(batch->t_len[i]), qs, ts, costs);
    });
    uint64_t used = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (used + res[i].cigar.size() > out->cigar_capacity) return PHR_ERR_CAPACITY;
        std::memcpy(out->cigar + used, res[i].cigar.data(), res[i].cigar.size());
        fill_alignment(res[i], &out->aln[i], used);
        used += res[i].cigar.size();
    }
    out->cigar_used = used;
    return PHR_OK;
}

// Timing helper for the CPU baseline: extends pairs [0, n) and discards the CIGARs,
// returning the sum of edit distances (so the work cannot be optimised away).
uint64_t orc_extend_batch_time(int32_t engine, const phr_pair_batch* batch, phr_affine_costs costs,
                               int32_t nthreads) {
    std::atomic<uint64_t> acc{0};
    parallel_for(batch->n_pairs, nthreads, [&](uint64_t i) {
        const uint8_t* q = batch->seq + batch->q_off[i];
        const uint8_t* t = batch->seq + batch->t_off[i];
        int32_t qs = batch->q_seed ? static_cast<int32_t>(batch->q_seed[i]) : 0;
        int32_t ts = batch->t_seed ? static_cast<int32_t>(batch->t_seed[i]) : 0;
        Aln a = extend_one(static_cast<phr_engine>(engine), q, static_cast<int32_t>(batch->q_len[i]), t,
                           static_cast<int32_t>(batch->t_len[i]), qs, ts, costs);
        acc.fetch_add(static_cast<uint64_t>(a.ed) + a.cigar.size());
    });
    return acc.load();
}

// Sketches sequence `s` into (values, positions); returns the count. Capacity must be
// at least max(len - k + 1, 0).
uint64_t orc_sketch(const uint8_t* s, uint64_t len, int32_t k, int32_t w, int32_t alphabet,
                    uint64_t* values, uint32_t* positions) {
    std::vector<std::pair<uint64_t, uint32_t>> sk;
    sketch_seq(s, static_cast<int64_t>(len), k, w, alphabet, &sk);
    for (size_t i = 0; i < sk.size(); ++i) {
        values[i] = sk[i].first;
        positions[i] = sk[i].second;
    }
    return sk.size();
}

// seed_occurrence_cap over an index built from (values, positions).
uint64_t orc_occurrence_cap(const uint64_t* values, const uint32_t* positions, uint64_t n, uint64_t floor) {
    std::vector<std::pair<uint64_t, uint32_t>> sk(n);
    for (uint64_t i = 0; i < n; ++i) sk[i] = {values[i], positions[i]};
    Index idx;
    build_index(sk, floor, &idx);
    return idx.cap;
}

// find_seeds_indexed_capped with an explicit cap (max_occ). Returns the seed count;
// writes up to `cap_out` seeds.
uint64_t orc_find_seeds(const uint64_t* tvals, const uint32_t* tpos, uint64_t tn, const uint64_t* qvals,
                        const uint32_t* qpos, uint64_t qn, uint64_t max_occ, phr_seed* out, uint64_t cap_out) {
    std::vector<std::pair<uint64_t, uint32_t>> tsk(tn), qsk(qn);
    for (uint64_t i = 0; i < tn; ++i) tsk[i] = {tvals[i], tpos[i]};
    for (uint64_t i = 0; i < qn; ++i) qsk[i] = {qvals[i], qpos[i]};
    Index idx;
    build_index(tsk, 256, &idx);
    idx.cap = max_occ;
    std::vector<SeedT> seeds = find_seeds(qsk, idx);
    for (uint64_t i = 0; i < seeds.size() && i < cap_out; ++i) {
        out[i].query_pos = seeds[i].qpos;
        out[i].target_pos = seeds[i].tpos;
        out[i].minimizer = seeds[i].val;
    }
    return seeds.size();
}

// chain_seeds with explicit parameters. Writes chains (seed_off into `seeds_out`).
// Returns the chain count, or -1 if an output buffer is too small.
int64_t orc_chain_seeds(const phr_seed* seeds, uint64_t n, int64_t seed_len, int64_t max_band,
                        int64_t max_dist_x, uint64_t max_iter, uint64_t max_skip, double gap_penalty,
                        int64_t min_chain_score, phr_chain* chains_out, uint64_t chain_cap_out,
                        phr_seed* seeds_out, uint64_t seed_cap_out) {
    std::vector<SeedT> in(n);
    for (uint64_t i = 0; i < n; ++i) in[i] = {seeds[i].query_pos, seeds[i].target_pos, seeds[i].minimizer};
    ChainParams p;
    p.seed_len = seed_len;
    p.max_band = max_band;
    p.max_dist_x = max_dist_x;
    p.max_iter = max_iter;
    p.max_skip = max_skip;
    p.gap_penalty = gap_penalty;
    p.min_chain_score = min_chain_score;
    std::vector<ChainT> ch = chain_seeds(in, p);
    if (ch.size() > chain_cap_out) return -1;
    uint64_t so = 0;
    for (size_t c = 0; c < ch.size(); ++c) {
        if (so + ch[c].seeds.size() > seed_cap_out) return -1;
        chains_out[c].score = ch[c].score;
        chains_out[c].seed_off = static_cast<uint32_t>(so);
        chains_out[c].n_seeds = static_cast<uint32_t>(ch[c].seeds.size());
        chains_out[c].target_start = ch[c].target_start();
        chains_out[c]._pad = 0;
        for (auto& s : ch[c].seeds) {
            seeds_out[so].query_pos = s.qpos;
            seeds_out[so].target_pos = s.tpos;
            seeds_out[so].minimizer = s.val;
            ++so;
        }
    }
    return static_cast<int64_t>(ch.size());
}

// score_alignments (lib.rs:170-199) over caller alignments (CIGARs in `cigar`).
// Writes the primary index and a 0/1 alternative flag per alignment. Returns -1 on
// an empty slice (the reference panics there), else 0.
int32_t orc_score_alignments(const phr_alignment* alns, const char* cigar, uint64_t n, uint64_t query_len,
                             uint64_t* primary_idx, uint8_t* is_alt) {
    if (n == 0) return -1;
    std::vector<Aln> v(n);
    for (uint64_t i = 0; i < n; ++i) {
        v[i].cigar.assign(cigar + alns[i].cigar_off, alns[i].cigar_len);
        v[i].ed = static_cast<int32_t>(alns[i].edit_distance);
        v[i].qs = static_cast<int32_t>(alns[i].query_start);
        v[i].qe = static_cast<int32_t>(alns[i].query_end);
        v[i].ts = static_cast<int32_t>(alns[i].target_start);
        v[i].te = static_cast<int32_t>(alns[i].target_end);
    }
    uint64_t pi = 0;
    for (uint64_t i = 1; i < n; ++i)
        if (v[i].ed < v[pi].ed) pi = i;
    Scored s = score_alignments(v, query_len);
    *primary_idx = pi;
    size_t ai = 0;
    for (uint64_t i = 0; i < n; ++i) {
        is_alt[i] = 0;
        if (ai < s.alts.size() && v[i] == s.alts[ai] && !(v[i] == s.primary)) {
            is_alt[i] = 1;
            ++ai;
        }
    }
    return 0;
}

// --- align_read over a target -------------------------------------------------
void* orc_target_create(const uint8_t* target, uint64_t len, int32_t alphabet) {
    Target* tg = new Target();
    tg->bytes.assign(target, target + len);
    tg->alphabet = alphabet;
    std::vector<std::pair<uint64_t, uint32_t>> sk;
    if (alphabet == PHR_ALPHABET_DNA)
        sketch_seq(target, static_cast<int64_t>(len), 21, 11, PHR_ALPHABET_DNA, &sk);
    else
        sketch_seq(target, static_cast<int64_t>(len), 6, 5, PHR_ALPHABET_PROTEIN, &sk);
    build_index(sk, 256, &tg->index);
    tg->repeats = detect_tandem_repeats(target, len, 3);
    return tg;
}

void orc_target_destroy(void* t) { delete static_cast<Target*>(t); }

uint64_t orc_target_cap(void* t) { return static_cast<Target*>(t)->index.cap; }

// align_read for each read; output layout matches phr_align_reads. Returns 0 or
// PHR_ERR_CAPACITY.
int32_t orc_align_reads(void* tgt, const phr_read_batch* reads, const phr_align_config* cfg,
                        phr_read_result_arena* out, phr_align_stats* stats, int32_t nthreads) {
    const Target& tg = *static_cast<Target*>(tgt);
    const uint64_t n = reads->n_reads;
    std::vector<ReadOut> res(n);
    parallel_for(n, nthreads, [&](uint64_t i) {
        std::vector<std::pair<uint64_t, uint32_t>> stored;
        const std::vector<std::pair<uint64_t, uint32_t>>* sp = nullptr;
        if (reads->has_stored && reads->has_stored[i]) {
            uint64_t o = reads->s_off[i];
            for (uint32_t j = 0; j < reads->s_n[i]; ++j)
                stored.push_back({reads->s_values[o + j], reads->s_positions[o + j]});
            sp = &stored;
        }
        align_read(tg, reads->seq + reads->off[i], reads->len[i], *cfg, sp, &res[i]);
    });
    uint64_t aused = 0, cused = 0;
    for (uint64_t i = 0; i < n; ++i) {
        ReadOut& r = res[i];
        phr_read_result& o = out->reads[i];
        std::memset(&o, 0, sizeof(o));
        o.outcome = r.outcome;
        o.has_result = r.has_result ? 1 : 0;
        o.reverse = r.reverse ? 1 : 0;
        o.aln_off = aused;
        if (stats) {
            uint64_t* b[] = {&stats->placed, &stats->no_seed, &stats->below_threshold, &stats->fast_cutoff,
                             &stats->no_alignment};
            *b[r.outcome] += 1;
        }
        if (!r.has_result) continue;
        std::vector<const Aln*> list{&r.scored.primary};
        for (auto& a : r.scored.alts) list.push_back(&a);
        if (aused + list.size() > out->aln_capacity) return PHR_ERR_CAPACITY;
        for (const Aln* a : list) {
            if (cused + a->cigar.size() > out->cigar_capacity) return PHR_ERR_CAPACITY;
            std::memcpy(out->cigar + cused, a->cigar.data(), a->cigar.size());
            fill_alignment(*a, &out->aln[aused], cused);
            cused += a->cigar.size();
            ++aused;
        }
        o.n_aln = static_cast<uint32_t>(list.size());
    }
    out->aln_used = aused;
    out->cigar_used = cused;
    return PHR_OK;
}

// Tandem repeats of `s` (min_repeat_count 3). Writes min(count, cap) regions; returns the count.
uint64_t orc_tandem_repeats(const uint8_t* s, uint64_t n, uint32_t* start, uint32_t* end, uint64_t cap) {
    std::vector<RepeatRegionT> r = detect_tandem_repeats(s, n, 3);
    for (uint64_t i = 0; i < r.size() && i < cap; ++i) {
        start[i] = static_cast<uint32_t>(r[i].start);
        end[i] = static_cast<uint32_t>(r[i].end);
    }
    return r.size();
}

// Variant observations of every read with a result in `res` (the layout phr_align_reads
// writes: primary first, then the alternatives), as align_read builds them
// (executor.rs:735-775). Output layout matches phr_align_reads_variants. Returns 0 or
// PHR_ERR_CAPACITY.
int32_t orc_variants(void* tgt, const phr_read_batch* reads, const phr_read_result_arena* res,
                     const phr_align_config* cfg, const phr_variant_config* vcfg, phr_variant_arena* vout) {
    const Target& tg = *static_cast<Target*>(tgt);
    const uint64_t n = reads->n_reads;
    size_t radius = vcfg && vcfg->coverage_radius ? vcfg->coverage_radius
                    : cfg->strategy == PHR_FAST   ? 150
                    : cfg->strategy == PHR_BALANCED ? 50
                                                    : 25;
    const uint32_t* hs = vcfg ? vcfg->hotspot_start : nullptr;
    const uint32_t* he = vcfg ? vcfg->hotspot_end : nullptr;
    const size_t nhs = vcfg && hs && he ? vcfg->n_hotspots : 0;
    const size_t tlen = tg.bytes.size();
    VariantOut out;
    for (uint64_t i = 0; i < n; ++i) {
        vout->read_variant_off[i] = out.v.size();
        const phr_read_result& r = res->reads[i];
        if (!r.has_result || r.n_aln == 0) continue;
        const uint8_t* read = reads->seq + reads->off[i];
        const size_t qlen = reads->len[i];
        std::vector<uint8_t> q = r.reverse ? revcomp(read, qlen) : std::vector<uint8_t>(read, read + qlen);
        std::vector<std::pair<size_t, size_t>> windows;
        for (uint32_t a = 0; a < r.n_aln; ++a) {
            const phr_alignment& x = res->aln[r.aln_off + a];
            const size_t s0 = std::min<size_t>(x.target_start, tlen), e0 = std::min<size_t>(x.target_end, tlen);
            if (s0 < e0) windows.push_back({s0, e0});
        }
        const phr_alignment& p = res->aln[r.aln_off];
        const std::string cig(res->cigar + p.cigar_off, p.cigar_len);
        const double score = 1.0 - static_cast<double>(p.edit_distance) / static_cast<double>(std::max<size_t>(qlen, 1));
        extract_variants(cig, p.target_start, q.data(), qlen, tg.bytes.data(), tlen, p.edit_distance, windows,
                         tg.repeats, hs, he, nhs, score, radius, r.reverse, static_cast<uint32_t>(i), &out);
    }
    vout->read_variant_off[n] = out.v.size();
    if (out.v.size() > vout->variant_capacity || out.cov.size() > vout->coverage_capacity ||
        out.al.size() > vout->allele_capacity)
        return PHR_ERR_CAPACITY;
    if (!out.v.empty()) std::memcpy(vout->variants, out.v.data(), out.v.size() * sizeof(phr_variant));
    if (!out.cov.empty()) std::memcpy(vout->coverage, out.cov.data(), out.cov.size() * 4);
    if (!out.al.empty()) std::memcpy(vout->alleles, out.al.data(), out.al.size() * sizeof(phr_allele));
    vout->variant_used = out.v.size();
    vout->coverage_used = out.cov.size();
    vout->allele_used = out.al.size();
    return PHR_OK;
}

// Coverage merge of merge_result (phraya-cli/src/main.rs:556-572) over alignment windows
// (compute_windowed_coverage, executor.rs:1071-1090: count 1 over [min(ts, len),
// min(te, len))), each window quantized by quantize_coverage (executor.rs:1092-1096)
// unless `depth`. Accumulates into track[0 .. tlen).
void orc_coverage_merge(const phr_alignment* aln, uint64_t n, uint64_t tlen, int32_t depth, uint32_t* track) {
    for (uint64_t a = 0; a < n; ++a) {
        const uint64_t s0 = std::min<uint64_t>(aln[a].target_start, tlen);
        const uint64_t e0 = std::min<uint64_t>(aln[a].target_end, tlen);
        for (uint64_t p = s0; p < e0; ++p) {
            const uint32_t c = 1;
            track[p] += depth ? c : ((c + 2) / 5) * 5;
        }
    }
}

// anchors_from_chains over chain target starts (in chain order); returns the anchor count.
uint64_t orc_anchors(const uint32_t* chain_starts, uint64_t n, int32_t strategy, uint32_t* out) {
    const std::vector<uint32_t> a = anchors_from_chains(std::vector<uint32_t>(chain_starts, chain_starts + n), strategy);
    for (size_t i = 0; i < a.size(); ++i) out[i] = a[i];
    return a.size();
}

}  // extern "C"
