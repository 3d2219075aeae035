// Link libneo_gpu.so (built in-tree by nightstream_b200/build.py).
fn main() {
    let dir = std::env::var("NEO_GPU_LIB_DIR").unwrap_or_else(|_| {
        let here = std::path::PathBuf::from(std::env::var("CARGO_MANIFEST_DIR").unwrap());
        here.join("../..").canonicalize().unwrap().to_string_lossy().into_owned()
    });
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=neo_gpu");
    println!("cargo:rerun-if-env-changed=NEO_GPU_LIB_DIR");
}
