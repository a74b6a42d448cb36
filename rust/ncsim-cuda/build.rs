//! Links libncsim_cuda.so, built by `python -m ncsim_b200.build` (nvcc,
//! sm_100a).  NCSIM_CUDA_LIB_DIR names the directory that holds it (default:
//! the package directory of this repository).
fn main() {
    let dir = std::env::var("NCSIM_CUDA_LIB_DIR").unwrap_or_else(|_| {
        let here = std::env::var("CARGO_MANIFEST_DIR").unwrap();
        format!("{here}/../../ncsim_b200")
    });
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=ncsim_cuda");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{dir}");
    println!("cargo:rerun-if-env-changed=NCSIM_CUDA_LIB_DIR");
}
