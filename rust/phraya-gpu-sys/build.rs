// Links libphraya_b200, either prebuilt (python -m phraya_b200.build) or compiled here
// from the CUDA sources with nvcc through `cc` (PHRAYA_B200_BUILD=1). The source list is
// phraya_b200/csrc/SOURCES, the same manifest the Python build reads.
use std::path::PathBuf;

fn main() {
    let root = std::env::var("PHRAYA_B200_DIR")
        .map(PathBuf::from)
        .unwrap_or_else(|_| PathBuf::from(env!("CARGO_MANIFEST_DIR")).join("../.."));
    let csrc = root.join("phraya_b200").join("csrc");
    let manifest = csrc.join("SOURCES");
    println!("cargo:rerun-if-changed={}", manifest.display());
    println!("cargo:rerun-if-changed={}", root.join("include").join("phraya_gpu.h").display());
    println!("cargo:rerun-if-env-changed=PHRAYA_B200_BUILD");
    if std::env::var("PHRAYA_B200_BUILD").is_ok() {
        let list = std::fs::read_to_string(&manifest).expect("phraya_b200/csrc/SOURCES");
        let files: Vec<PathBuf> = list
            .lines()
            .map(str::trim)
            .filter(|l| !l.is_empty() && !l.starts_with('#'))
            .map(|l| csrc.join(l))
            .collect();
        for f in &files {
            println!("cargo:rerun-if-changed={}", f.display());
        }
        cc::Build::new()
            .cuda(true)
            .cudart("shared")
            .flag("-gencode")
            .flag("arch=compute_100a,code=sm_100a")
            .flag("-O3")
            .flag("-std=c++17")
            .flag("--expt-relaxed-constexpr")
            .files(files)
            .compile("phraya_b200");
        println!("cargo:rustc-link-lib=dylib=stdc++");
    } else {
        println!("cargo:rustc-link-search=native={}", root.join("phraya_b200").display());
        println!("cargo:rustc-link-lib=dylib=phraya_b200");
    }
}
