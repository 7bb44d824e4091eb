// Link libsxhmm.so.  SXHMM_LIB_DIR names the directory that holds it (by
// default the package's own sxhmm/ directory, two levels up from this crate,
// where sentinel-x_b200/build.py writes it).
use std::env;
use std::path::PathBuf;

fn main() {
    let dir = match env::var("SXHMM_LIB_DIR") {
        Ok(d) => PathBuf::from(d),
        Err(_) => PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap()).join("../../sxhmm"),
    };
    println!("cargo:rustc-link-search=native={}", dir.display());
    println!("cargo:rustc-link-lib=dylib=sxhmm");
    println!("cargo:rerun-if-env-changed=SXHMM_LIB_DIR");
}
