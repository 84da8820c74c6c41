"""Writes tests/golden/case2_digests.json: digests of the reference's own read simulator's
output, used to pin phraya_b200.casegen's restatement of it.

Runs only where the reference tree is present (it is read, never copied):
  python tests/golden/make_case2_digests.py /root/reference

For each parameter set it runs scripts/benchmark/local/gen_synthetic.py into a scratch
folder and records SHA-256 digests of the genome sequence, of the reads joined by
newlines, and of the truth rows (start, strand, substitutions, indel events). It also
imports the simulator's mutation function and records digests of its output on fixed
protein fragments and seeds (the protein generator reuses that function with the
20-residue alphabet).
"""
import hashlib
import importlib.util
import json
import os
import random
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SCRATCH = os.path.join(HERE, "..", "..", "_work", "case2_digests")

PARAM_SETS = [
    # the short-read benchmark case: 1 Mbp genome, 20,000 x 150 bp reads
    {"genome_size": 1_000_000, "num_reads": 20_000, "read_len": 150, "divergence": 0.01, "indel_rate": 0.0005,
     "indel_max_len": 3, "seed": 0},
    {"genome_size": 5000, "num_reads": 300, "read_len": 100, "divergence": 0.05, "indel_rate": 0.02,
     "indel_max_len": 5, "seed": 7},
    {"genome_size": 3000, "num_reads": 60, "read_len": 80, "divergence": 0.03, "indel_rate": 0.0,
     "indel_max_len": 5, "seed": 1},
]

AMINO_ACIDS = "ACDEFGHIKLMNPQRSTVWY"
PROTEIN_CASES = [(300, 0.30, 0.0, 3, 11), (500, 0.02, 0.01, 3, 12), (150, 0.10, 0.05, 5, 13)]


def sha(s):
    return hashlib.sha256(s.encode()).hexdigest()


def read_fasta(path):
    with open(path) as fh:
        return "".join(ln.strip() for ln in fh if not ln.startswith(">"))


def read_fastq(path):
    with open(path) as fh:
        lines = fh.read().split("\n")
    return [lines[i + 1] for i in range(0, len(lines) - 1, 4)]


def read_truth(path):
    with open(path) as fh:
        rows = fh.read().rstrip("\n").split("\n")[1:]
    return [r.split("\t", 1)[1] for r in rows]  # drop read_id


def main(ref_root):
    script = os.path.join(ref_root, "scripts", "benchmark", "local", "gen_synthetic.py")
    os.makedirs(SCRATCH, exist_ok=True)
    out = {"generator": "scripts/benchmark/local/gen_synthetic.py", "sets": [], "protein_mutations": []}
    for p in PARAM_SETS:
        fa, fq = os.path.join(SCRATCH, "ref.fa"), os.path.join(SCRATCH, "reads.fq")
        cmd = [sys.executable, script, "--genome-size", str(p["genome_size"]), "--num-reads", str(p["num_reads"]),
               "--read-len", str(p["read_len"]), "--divergence", str(p["divergence"]),
               "--indel-rate", str(p["indel_rate"]), "--indel-max-len", str(p["indel_max_len"]),
               "--seed", str(p["seed"]), "--ref-out", fa, "--reads-out", fq]
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
        reads = read_fastq(fq)
        out["sets"].append({"params": p, "genome_sha256": sha(read_fasta(fa)), "reads_sha256": sha("\n".join(reads)),
                            "truth_sha256": sha("\n".join(read_truth(fq + ".truth.tsv"))),
                            "n_reads": len(reads)})
    spec = importlib.util.spec_from_file_location("ref_gen_synthetic", script)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    for length, div, indel, maxlen, seed in PROTEIN_CASES:
        rng = random.Random(seed)
        frag = "".join(rng.choices(AMINO_ACIDS, k=length))
        mut, n_subs, ev = mod.mutate_with_truth(frag, div, indel, maxlen, rng, alphabet=AMINO_ACIDS)
        out["protein_mutations"].append({"length": length, "divergence": div, "indel_rate": indel,
                                         "indel_max_len": maxlen, "seed": seed, "mutated_sha256": sha(mut),
                                         "n_subs": n_subs, "events": [list(e) for e in ev]})
    shutil.rmtree(SCRATCH)
    with open(os.path.join(HERE, "case2_digests.json"), "w") as fh:
        json.dump(out, fh, indent=1)
        fh.write("\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
