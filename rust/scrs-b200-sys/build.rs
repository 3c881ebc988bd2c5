// Links libscrs_b200.so; SCRS_B200_LIB_DIR names its directory
// (scrs_b200/_lib after `python -m scrs_b200.build`).
fn main() {
    let dir = std::env::var("SCRS_B200_LIB_DIR").expect("SCRS_B200_LIB_DIR: directory of libscrs_b200.so");
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=scrs_b200");
    println!("cargo:rerun-if-env-changed=SCRS_B200_LIB_DIR");
}
