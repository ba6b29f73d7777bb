// Links libfgfcuda.so, built in-tree by `python -m fgf_b200.build` (nvcc for
// sm_100a). FGF_CUDA_LIB_DIR names the directory holding it; by default the
// package directory two levels up (fgf_b200/).
fn main() {
    let dir = std::env::var("FGF_CUDA_LIB_DIR")
        .unwrap_or_else(|_| format!("{}/../..", env!("CARGO_MANIFEST_DIR")));
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=fgfcuda");
    println!("cargo:rerun-if-env-changed=FGF_CUDA_LIB_DIR");
}
