"""Seeded generators and independent checkers restated from phraya's own tests.

Every generator reproduces the reference's fixture bit-for-bit from the same seed (the
RNG recurrences are cited), so the oracle and the CUDA engine are checked on exactly the
inputs phraya's test-suite uses. The O(nm) checkers are independent of every WFA/Myers
implementation under test.
"""
import re

M64 = (1 << 64) - 1
LCG_A = 6364136223846793005
LCG_C = 1442695040888963407


class SplitMix64:
    """`Rng` of phraya-align/src/wfa_simd.rs:2999-3009."""

    def __init__(self, state):
        self.s = state & M64

    def next(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & M64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return z ^ (z >> 31)

    def below(self, n):
        return self.next() % n


def random_dna(rng, n):
    """wfa_simd.rs:3010-3013."""
    return bytes(b"ACGT"[rng.below(4)] for _ in range(n))


def diverge_dna(rng, seq, rate_pct):
    """wfa_simd.rs:3014-3026."""
    out = bytearray()
    for b in seq:
        if rng.below(100) < rate_pct:
            r = rng.below(3)
            if r == 0:
                out.append(b"ACGT"[rng.below(4)])
            elif r == 1:
                pass
            else:
                out.append(b"ACGT"[rng.below(4)])
                out.append(b)
        else:
            out.append(b)
    return bytes(out)


def scalar_edit_sweep():
    """Inputs of edit_distance_matches_scalar_property (wfa_simd.rs:3028-3051)."""
    rng = SplitMix64(0xDEAD_BEEF_1234)
    cases = []
    for ql in [0, 1, 4, 8, 16, 32, 64, 128]:
        for dv in [0, 2, 10, 30]:
            for _ in range(10):
                q = random_dna(rng, ql)
                t = diverge_dna(rng, q, dv)
                cases.append((q, t))
    return cases


def lcg_bytes(n, alphabet, seed):
    """lcg_bytes of wfa_simd.rs:3233-3242."""
    x = seed & M64
    out = bytearray()
    for _ in range(n):
        x = (x * LCG_A + LCG_C) & M64
        out.append(alphabet[((x >> 33) % len(alphabet))])
    return bytes(out)


def affine_fitting_cases():
    """Inputs of affine_score_matches_gotoh_oracle_across_random_cases (wfa_simd.rs:3314-3371)."""
    AA = b"ACGT"
    cases = []
    for seed in range(60):
        qlen = 20 + seed % 15
        q = lcg_bytes(qlen, AA, seed * 31 + 7)
        t = bytearray()
        x = (seed + 99) & M64
        qi = 0
        while qi < len(q):
            x = (x * LCG_A + LCG_C) & M64
            roll = (x >> 40) % 100
            if roll < 8:
                ln = 1 + (x >> 20) % 3
                for _ in range(ln):
                    x = (x * LCG_A + 1) & M64
                    t.append(AA[(x >> 4) % 4])
            elif roll < 16 and qi + 1 < len(q):
                qi += 1
            elif roll < 30:
                x = (x * LCG_A + 1) & M64
                t.append(AA[(x >> 4) % 4])
                qi += 1
            else:
                t.append(q[qi])
                qi += 1
        t += lcg_bytes(len(q) + 20, AA, seed * 13 + 500)
        cases.append((q, bytes(t)))
    return cases


def affine_global_cases():
    """Inputs of affine_score_matches_gotoh_oracle_in_global_mode (wfa_simd.rs:3401-3454)."""
    AA = b"ACGT"
    cases = []
    for seed in range(40):
        qlen = 15 + seed % 10
        q = lcg_bytes(qlen, AA, seed * 41 + 3)
        t = bytearray()
        x = (seed + 7) & M64
        qi = 0
        while qi < len(q):
            x = (x * LCG_A + LCG_C) & M64
            roll = (x >> 40) % 100
            if roll < 6 and len(t) + 2 < len(q) + 5:
                x = (x * LCG_A + 1) & M64
                t.append(AA[(x >> 4) % 4])
            elif roll < 12 and qi + 1 < len(q):
                qi += 1
            elif roll < 25:
                x = (x * LCG_A + 1) & M64
                t.append(AA[(x >> 4) % 4])
                qi += 1
            else:
                t.append(q[qi])
                qi += 1
        cases.append((q, bytes(t)))
    return cases


def myers_wfa_fitting_sweep():
    """Inputs of issue_176_myers_fitting_edit_distance_matches_wfa_sweep
    (phraya-align/tests/test_wfa_algorithm.rs:375-436)."""
    state = [0x9E3779B97F4A7C15]

    def nxt():
        state[0] = (state[0] * LCG_A + LCG_C) & M64
        return state[0] >> 33

    bases = b"ACGT"
    cases = []
    for query_len in [60, 120, 200, 350]:
        for trial in range(80):
            query = bytes(bases[nxt() % 4] for _ in range(query_len))
            region = bytearray(query)
            num_snps = nxt() % 5
            for _ in range(num_snps):
                if not region:
                    break
                p = nxt() % len(region)
                region[p] = bases[nxt() % 4]
            m = trial % 3
            if m == 1 and len(region) > 10:
                p = nxt() % (len(region) - 4)
                d = 1 + nxt() % 3
                del region[p:min(p + d, len(region))]
            elif m == 2:
                p = nxt() % (len(region) + 1)
                ins = 1 + nxt() % 3
                extra = bytes(bases[nxt() % 4] for _ in range(ins))
                region[p:p] = extra
            tail_len = query_len + query_len // 2 + 20
            tail = bytes(bases[nxt() % 4] for _ in range(tail_len))
            cases.append((query, bytes(region) + tail))
    return cases


def lcp_battery():
    """battery() of phraya-align/src/wfa_simd.rs:3831-3853."""
    cases = []
    for ln in range(40):
        v = bytes(b"ACGT"[i % 4] for i in range(ln))
        cases.append((v, v))
    for p in range(40):
        a = bytes(b"ACGT"[i % 4] for i in range(40))
        b = bytearray(a)
        b[p] ^= 0x01
        cases.append((a, bytes(b)))
    cases.append((b"ACGTACGTAC", b"ACGTACGT"))
    cases.append((b"ACGT", b"ACGTACGTACGT"))
    cases.append((b"", b"ACGT"))
    cases.append((b"ACGT", b""))
    return cases


def diverse_dna(n, seed):
    """diverse_dna of phraya-align/tests/chaining_correctness.rs:29-37."""
    x = seed & M64
    out = bytearray()
    for _ in range(n):
        x = (x * LCG_A + LCG_C) & M64
        out.append(b"ACGT"[(x >> 33) & 3])
    return bytes(out)


AMINO = b"ACDEFGHIKLMNPQRSTVWY"


def diverse_protein(n, seed):
    """diverse_protein of phraya-align/src/executor.rs:1949-1960 (tests module)."""
    x = seed & M64
    out = bytearray()
    for _ in range(n):
        x = (x * LCG_A + LCG_C) & M64
        out.append(AMINO[(x >> 33) % 20])
    return bytes(out)


def protein_wfa_myers_cases():
    """The 20 query/target pairs of protein_wfa_myers_edit_distance_agree
    (executor.rs:2001-2027): query diverse_protein(120, 97 s + 1), target = query with
    substitutions at (s % 5) * 15 % of positions drawn from its own LCG."""
    cases = []
    for seed in range(20):
        q = diverse_protein(120, seed * 97 + 1)
        t = bytearray(q)
        rate = seed % 5
        x = (seed + 12345) & M64
        for i in range(len(t)):
            x = (x * LCG_A + LCG_C) & M64
            if (x >> 40) % 100 < rate * 15:
                x = (x * LCG_A + 1) & M64
                t[i] = AMINO[(x >> 33) % 20]
        cases.append((q, bytes(t)))
    return cases


# ---------------------------------------------------------------------------
# Independent checkers
# ---------------------------------------------------------------------------
def edit_distance_dp(q, t):
    """Global unit-cost edit distance (fill_scalar, wfa_simd.rs:1138-1160)."""
    prev = list(range(len(t) + 1))
    for i in range(1, len(q) + 1):
        cur = [i] + [0] * len(t)
        qi = q[i - 1]
        for j in range(1, len(t) + 1):
            cost = 0 if qi == t[j - 1] else 1
            cur[j] = min(prev[j] + 1, cur[j - 1] + 1, prev[j - 1] + cost)
        prev = cur
    return prev[len(t)]


def gotoh(q, t, costs, fitting):
    """Gotoh affine DP (wfa_simd.rs:3118-3170 fitting, :3458-3493 global), score only."""
    x, o, e = costs
    INF = 1 << 40
    qn, tn = len(q), len(t)
    M = [[INF] * (tn + 1) for _ in range(qn + 1)]
    I = [[INF] * (tn + 1) for _ in range(qn + 1)]
    D = [[INF] * (tn + 1) for _ in range(qn + 1)]
    M[0][0] = 0
    for i in range(1, qn + 1):
        I[i][0] = o + e * i
    for j in range(1, tn + 1):
        D[0][j] = o + e * j
    for i in range(1, qn + 1):
        for j in range(1, tn + 1):
            sub = 0 if q[i - 1] == t[j - 1] else x
            M[i][j] = min(M[i - 1][j - 1], I[i - 1][j - 1], D[i - 1][j - 1]) + sub
            em_up = min(M[i - 1][j], I[i - 1][j], D[i - 1][j])
            em_left = min(M[i][j - 1], I[i][j - 1], D[i][j - 1])
            I[i][j] = min(em_up + o + e, I[i - 1][j] + e)
            D[i][j] = min(em_left + o + e, D[i][j - 1] + e)
    if fitting:
        return min(min(M[qn][j], I[qn][j], D[qn][j]) for j in range(tn + 1))
    return min(M[qn][tn], I[qn][tn], D[qn][tn])


CIGAR_RE = re.compile(r"(\d+)([MXID])")


def cigar_ops(cigar):
    ops = [(int(n), op) for n, op in CIGAR_RE.findall(cigar)]
    assert "".join(f"{n}{op}" for n, op in ops) == cigar, f"malformed CIGAR {cigar!r}"
    return ops


def cigar_affine_cost(cigar, costs):
    """cigar_affine_cost (wfa_simd.rs:3175-3192)."""
    x, o, e = costs
    c = 0
    for n, op in cigar_ops(cigar):
        if op == "X":
            c += n * x
        elif op in "ID":
            c += o + n * e
    return c


def replay(cigar, q, t):
    """assert_cigar_replays_correctly (wfa_simd.rs:3198-3231) minus the final length
    asserts; returns (query consumed, target consumed)."""
    qi = ti = 0
    for n, op in cigar_ops(cigar):
        if op == "M":
            for _ in range(n):
                assert q[qi] == t[ti], f"M at q[{qi}]/t[{ti}] is not a match"
                qi += 1
                ti += 1
        elif op == "X":
            for _ in range(n):
                assert q[qi] != t[ti], f"X at q[{qi}]/t[{ti}] is not a mismatch"
                qi += 1
                ti += 1
        elif op == "D":
            qi += n
        else:
            ti += n
    return qi, ti


def levenshtein_from_cigar(cigar):
    return sum(n for n, op in cigar_ops(cigar) if op != "M")
