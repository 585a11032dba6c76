// Links libfieldgrid.so (built by `python -m fieldgrid_b200.build`); FIELDGRID_LIB_DIR names the
// directory that holds it, and the CUDA runtime comes from CUDA_HOME (default /usr/local/cuda).
fn main() {
    if let Ok(dir) = std::env::var("FIELDGRID_LIB_DIR") {
        println!("cargo:rustc-link-search=native={dir}");
    }
    let cuda = std::env::var("CUDA_HOME").unwrap_or_else(|_| "/usr/local/cuda".into());
    println!("cargo:rustc-link-search=native={cuda}/lib64");
    println!("cargo:rustc-link-lib=dylib=fieldgrid");
    println!("cargo:rustc-link-lib=dylib=cudart");
    println!("cargo:rerun-if-env-changed=FIELDGRID_LIB_DIR");
}
