//! Builds libllr_b200.so with nvcc (sm_100a) through the package Makefile one directory up and
//! links it.  `LLR_B200_SKIP_BUILD=1` links a library built beforehand; `CUDA_HOME` (default
//! /usr/local/cuda) locates the CUDA runtime and cuFFT the library depends on.
use std::env;
use std::path::PathBuf;
use std::process::Command;

fn main() {
    let manifest = PathBuf::from(env::var("CARGO_MANIFEST_DIR").expect("cargo sets CARGO_MANIFEST_DIR"));
    let pkg = manifest.parent().expect("the crate lives in llr-reco_b200/rust").to_path_buf();
    for dep in ["csrc", "Makefile", "../include"] {
        println!("cargo:rerun-if-changed={}", pkg.join(dep).display());
    }
    println!("cargo:rerun-if-env-changed=LLR_B200_SKIP_BUILD");
    println!("cargo:rerun-if-env-changed=CUDA_HOME");
    if env::var_os("LLR_B200_SKIP_BUILD").is_none() {
        let jobs = env::var("NUM_JOBS").unwrap_or_else(|_| "8".to_string());
        let status = Command::new("make")
            .arg("-C")
            .arg(&pkg)
            .arg("-j")
            .arg(&jobs)
            .status()
            .expect("running make (nvcc, make and a C++ compiler are required)");
        assert!(status.success(), "building libllr_b200.so failed");
    }
    let cuda = env::var("CUDA_HOME").unwrap_or_else(|_| "/usr/local/cuda".to_string());
    println!("cargo:rustc-link-search=native={}", pkg.display());
    println!("cargo:rustc-link-search=native={}/lib64", cuda);
    println!("cargo:rustc-link-lib=dylib=llr_b200");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", pkg.display());
}
