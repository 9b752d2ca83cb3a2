// Links libgalaxy_bh.so, built in-tree by `python -m galaxy_b200.build`
// (nvcc, sm_100a).  GALAXY_BH_LIB_DIR overrides the directory; by default it
// is the package directory one level up from this crate.
use std::env;
use std::path::PathBuf;

fn main() {
    let dir = env::var("GALAXY_BH_LIB_DIR").map(PathBuf::from).unwrap_or_else(|_| {
        PathBuf::from(env::var("CARGO_MANIFEST_DIR").expect("cargo sets CARGO_MANIFEST_DIR"))
            .join("..")
    });
    println!("cargo:rerun-if-env-changed=GALAXY_BH_LIB_DIR");
    println!("cargo:rustc-link-search=native={}", dir.display());
    println!("cargo:rustc-link-lib=dylib=galaxy_bh");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", dir.display());
}
