//! Rust binding of libsxhmm, the B200 hmmsearch engine.
//!
//! `ffi` mirrors `include/sxhmm.h` one to one (the structs are `#[repr(C)]`
//! with the header's field order).  The safe layer above it owns the
//! library's objects (`Engine`, `ProfileSet`, `TargetSet`) and frees them on
//! drop; `Engine::search` is the device replacement of the reference's
//! `search_profiles` (src/hmmer/search.rs:213-234) and returns hits in the
//! same order (profile order, then target order, search.rs:225-232).
//!
//! The adapter from the reference's own types (`Profile`, `Targets`,
//! `SearchConfig`, `Hit`) to this crate is a short module on the reference's
//! side, selected by its `--gpu` flag (src/main.rs:424, src/pipeline.rs:102-104).

use std::ffi::{CStr, CString};
use std::os::raw::{c_char, c_int};
use std::path::Path;
use std::ptr::{null, null_mut};

#[allow(non_camel_case_types)]
pub mod ffi {
    use std::os::raw::{c_char, c_int};

    pub const SX_OK: c_int = 0;
    pub const SX_EINVAL: c_int = 1;
    pub const SX_ECUTOFF: c_int = 2;
    pub const SX_ENOMEM: c_int = 3;
    pub const SX_ECUDA: c_int = 4;
    pub const SX_ETIMEOUT: c_int = 5;
    pub const SX_EIO: c_int = 6;

    pub const SX_CUT_EVALUE: i32 = 0;
    pub const SX_CUT_BITS: i32 = 1;
    pub const SX_CUT_GA: i32 = 2;
    pub const SX_CUT_NC: i32 = 3;
    pub const SX_CUT_TC: i32 = 4;

    pub const SX_FLAG_PLAIN: u32 = 1;
    pub const SX_FLAG_ENV_DEVICE: u32 = 2;
    pub const SX_FLAG_ENV_HOST: u32 = 4;
    pub const SX_FLAG_TRACE_HOST: u32 = 8;
    pub const SX_FLAG_TRACE_DEVICE: u32 = 16;
    pub const SX_FLAG_NO_PRESCREEN: u32 = 32;

    #[repr(C)]
    pub struct sx_engine {
        _opaque: [u8; 0],
    }
    #[repr(C)]
    pub struct sx_profiles {
        _opaque: [u8; 0],
    }
    #[repr(C)]
    pub struct sx_targets {
        _opaque: [u8; 0],
    }
    #[repr(C)]
    pub struct sx_hits {
        _opaque: [u8; 0],
    }

    #[repr(C)]
    #[derive(Clone, Copy, Debug, Default)]
    pub struct sx_opts {
        pub device: i32,
        pub host_threads: i32,
        pub flags: u32,
        pub pipeline_blocks: i32,
        pub batch_bytes: i64,
    }

    #[repr(C)]
    #[derive(Clone, Copy, Debug)]
    pub struct sx_search_cfg {
        pub cutoff_kind: i32,
        pub filters: i32,
        pub null2: i32,
        pub reserved: i32,
        pub seq_threshold: f64,
        pub dom_threshold: f64,
        pub f1: f64,
        pub f2: f64,
        pub f3: f64,
        pub z: f64,
    }

    #[repr(C)]
    #[derive(Clone, Copy, Debug)]
    pub struct sx_hit {
        pub profile_index: i32,
        pub target_index: i32,
        pub qlen: i32,
        pub tlen: i32,
        pub score: f32,
        pub bias: f32,
        pub evalue: f64,
        pub nexpected: f32,
        pub ndomains: i32,
        pub domain_offset: i32,
        pub reserved: i32,
    }

    #[repr(C)]
    #[derive(Clone, Copy, Debug)]
    pub struct sx_domain {
        pub score: f32,
        pub bias: f32,
        pub c_evalue: f64,
        pub i_evalue: f64,
        pub hmm_from: i32,
        pub hmm_to: i32,
        pub ali_from: i32,
        pub ali_to: i32,
        pub env_from: i32,
        pub env_to: i32,
        pub reported: i32,
        pub reserved: i32,
    }

    #[repr(C)]
    #[derive(Clone, Copy, Debug)]
    pub struct sx_profile_info {
        pub name: *const c_char,
        pub acc: *const c_char,
        pub desc: *const c_char,
        pub m: i32,
        pub calibrated: i32,
        pub ga: [f32; 2],
        pub tc: [f32; 2],
        pub nc: [f32; 2],
        pub msv: [f64; 2],
        pub viterbi: [f64; 2],
        pub forward: [f64; 2],
    }

    #[repr(C)]
    #[derive(Clone, Copy, Debug)]
    pub struct sx_profile_arrays {
        pub name: *const c_char,
        pub acc: *const c_char,
        pub desc: *const c_char,
        pub m: i32,
        pub has_cutoffs: i32,
        pub msc: *const f32,
        pub mo: *const f32,
        pub t: *const f32,
        pub p: *const f32,
        pub compo: *const f32,
        pub msv_tbm: f32,
        pub ga: [f32; 2],
        pub tc: [f32; 2],
        pub nc: [f32; 2],
        pub has_stats: i32,
        pub msv: [f64; 2],
        pub viterbi: [f64; 2],
        pub forward: [f64; 2],
    }

    #[repr(C)]
    #[derive(Clone, Copy, Debug)]
    pub struct sx_search_stats {
        pub pairs_in: [i64; 8],
        pub pairs_out: [i64; 8],
        pub cells: [f64; 8],
        pub ms: [f64; 8],
        pub kernel_launches: i64,
        pub prescreen_pairs_in: i64,
        pub prescreen_pairs_out: i64,
        pub prescreen_cells: f64,
        pub prescreen_ms: f64,
        pub rescore_ms: f64,
        pub vprescreen_pairs_in: i64,
        pub vprescreen_pairs_out: i64,
        pub vprescreen_cells: f64,
        pub vprescreen_ms: f64,
    }

    extern "C" {
        pub fn sx_create(opts: *const sx_opts, out: *mut *mut sx_engine) -> c_int;
        pub fn sx_destroy(e: *mut sx_engine);
        pub fn sx_last_error() -> *const c_char;

        pub fn sx_profiles_load_file(e: *mut sx_engine, path: *const c_char, out: *mut *mut sx_profiles) -> c_int;
        pub fn sx_profiles_load_text(e: *mut sx_engine, text: *const c_char, len: usize, source: *const c_char,
                                     out: *mut *mut sx_profiles) -> c_int;
        pub fn sx_profiles_from_arrays(e: *mut sx_engine, profiles: *const sx_profile_arrays, n: usize,
                                       out: *mut *mut sx_profiles) -> c_int;
        pub fn sx_profiles_save(p: *const sx_profiles, path: *const c_char) -> c_int;
        pub fn sx_profiles_load_binary(e: *mut sx_engine, path: *const c_char, out: *mut *mut sx_profiles) -> c_int;
        pub fn sx_profiles_count(p: *const sx_profiles) -> i32;
        pub fn sx_profiles_info(p: *const sx_profiles, i: i32, out: *mut sx_profile_info) -> c_int;
        pub fn sx_profiles_free(p: *mut sx_profiles);

        pub fn sx_targets_create(e: *mut sx_engine, ids: *const *const c_char, seqs: *const *const u8,
                                 lens: *const usize, n: usize, out: *mut *mut sx_targets) -> c_int;
        pub fn sx_targets_create_digital(e: *mut sx_engine, dsq: *const u8, offsets: *const i64, lens: *const i64,
                                         n: usize, out: *mut *mut sx_targets) -> c_int;
        pub fn sx_targets_count(t: *const sx_targets) -> i64;
        pub fn sx_targets_free(t: *mut sx_targets);

        pub fn sx_search(e: *mut sx_engine, p: *const sx_profiles, t: *const sx_targets, cfg: *const sx_search_cfg,
                         out: *mut *mut sx_hits) -> c_int;
        pub fn sx_search_many(e: *mut sx_engine, sets: *const *const sx_profiles, n: usize, t: *const sx_targets,
                              cfg: *const sx_search_cfg, out: *mut *mut sx_hits) -> c_int;
        pub fn sx_hits_count(h: *const sx_hits) -> usize;
        pub fn sx_hits_array(h: *const sx_hits) -> *const sx_hit;
        pub fn sx_hits_domain_count(h: *const sx_hits) -> usize;
        pub fn sx_hits_domains(h: *const sx_hits) -> *const sx_domain;
        pub fn sx_hits_free(h: *mut sx_hits);
        pub fn sx_last_search_stats(e: *const sx_engine, out: *mut sx_search_stats) -> c_int;

        pub fn sx_shape_count(kind: c_int) -> c_int;
        pub fn sx_shape_info(kind: c_int, index: c_int, g: *mut i32, c: *mut i32, rt: *mut i32) -> c_int;
        pub fn sx_shape_for(e: *const sx_engine, kind: c_int, m: i32) -> c_int;
        pub fn sx_set_shape_table(e: *mut sx_engine, kind: c_int, shape_by_m: *const i32, len: usize) -> c_int;

        pub fn sx_score_pairs(e: *mut sx_engine, p: *const sx_profiles, t: *const sx_targets,
                              pair_profile: *const i32, pair_target: *const i32, npairs: usize, msv: *mut f32,
                              viterbi: *mut f32, forward: *mut f32, backward: *mut f32, bias: *mut f32) -> c_int;
        pub fn sx_score_prescreens(e: *mut sx_engine, p: *const sx_profiles, t: *const sx_targets,
                                   pair_profile: *const i32, pair_target: *const i32, npairs: usize,
                                   msv_bound: *mut f32, fwd_scan: *mut f32, vit_bound: *mut f32) -> c_int;
        pub fn sx_posterior_grad(e: *mut sx_engine, p: *const sx_profiles, t: *const sx_targets,
                                 pair_profile: *const i32, pair_target: *const i32, npairs: usize, m: i32,
                                 d_msc: *mut f32, d_isc: *mut f32, d_trans: *mut f32, lnz: *mut f64) -> c_int;
        pub fn sx_score_viterbi_static(e: *mut sx_engine, p: *const sx_profiles, t: *const sx_targets,
                                       pair_profile: *const i32, pair_target: *const i32, npairs: usize,
                                       viterbi: *mut f32) -> c_int;
    }
}

/// An error of the library: its class (`ffi::SX_E*`) and the message of
/// `sx_last_error`, whose texts are the reference's where callers match on
/// them (e.g. "GA bit thresholds unavailable on model X", search.rs:137).
#[derive(Debug, Clone)]
pub struct Error {
    pub code: c_int,
    pub message: String,
}

impl std::fmt::Display for Error {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        write!(f, "{}", self.message)
    }
}

impl std::error::Error for Error {}

pub type Result<T> = std::result::Result<T, Error>;

fn check(rc: c_int) -> Result<()> {
    if rc == ffi::SX_OK {
        return Ok(());
    }
    let message = unsafe { CStr::from_ptr(ffi::sx_last_error()) }.to_string_lossy().into_owned();
    Err(Error { code: rc, message })
}

fn cstring(s: &str) -> Result<CString> {
    CString::new(s).map_err(|_| Error { code: ffi::SX_EINVAL, message: format!("string contains NUL: {s:?}") })
}

/// `Cutoff` (src/hmmer/search.rs:26-38).
#[derive(Clone, Copy, Debug)]
pub enum Cutoff {
    Evalue { seq: f64, dom: f64 },
    Bits { seq: f64, dom: f64 },
    Gathering,
    Noise,
    Trusted,
}

/// `SearchConfig` + `PipelineConfig` (src/hmmer/search.rs:42-47,
/// src/hmmer/pipeline.rs:27-42), HMMER's defaults in `Default`.
#[derive(Clone, Copy, Debug)]
pub struct SearchConfig {
    pub cutoff: Cutoff,
    pub filters: bool,
    pub null2: bool,
    pub f1: f64,
    pub f2: f64,
    pub f3: f64,
    pub z: Option<f64>,
}

impl Default for SearchConfig {
    fn default() -> Self {
        SearchConfig { cutoff: Cutoff::Evalue { seq: 10.0, dom: 10.0 }, filters: true, null2: true, f1: 0.02,
                       f2: 1e-3, f3: 1e-5, z: None }
    }
}

impl SearchConfig {
    pub fn to_c(&self) -> ffi::sx_search_cfg {
        let (kind, seq, dom) = match self.cutoff {
            Cutoff::Evalue { seq, dom } => (ffi::SX_CUT_EVALUE, seq, dom),
            Cutoff::Bits { seq, dom } => (ffi::SX_CUT_BITS, seq, dom),
            Cutoff::Gathering => (ffi::SX_CUT_GA, 0.0, 0.0),
            Cutoff::Noise => (ffi::SX_CUT_NC, 0.0, 0.0),
            Cutoff::Trusted => (ffi::SX_CUT_TC, 0.0, 0.0),
        };
        ffi::sx_search_cfg { cutoff_kind: kind, filters: self.filters as i32, null2: self.null2 as i32, reserved: 0,
                             seq_threshold: seq, dom_threshold: dom, f1: self.f1, f2: self.f2, f3: self.f3,
                             z: self.z.unwrap_or(f64::NAN) }
    }
}

/// `DomainHit` (src/hmmer/search.rs:84-97); coordinates are 1-based inclusive.
#[derive(Clone, Debug, PartialEq)]
pub struct DomainHit {
    pub score: f32,
    pub bias: f32,
    pub c_evalue: f64,
    pub i_evalue: f64,
    pub hmm_from: usize,
    pub hmm_to: usize,
    pub ali_from: usize,
    pub ali_to: usize,
    pub env_from: usize,
    pub env_to: usize,
    pub reported: bool,
}

/// `Hit` (src/hmmer/search.rs:101-116) by index: the caller maps
/// `profile_index` / `target_index` back to its own names.
#[derive(Clone, Debug, PartialEq)]
pub struct Hit {
    pub profile_index: usize,
    pub target_index: usize,
    pub qlen: usize,
    pub tlen: usize,
    pub score: f32,
    pub bias: f32,
    pub evalue: f64,
    pub nexpected: f32,
    pub domains: Vec<DomainHit>,
}

/// One engine per device; calls on it are serialised by the library.
pub struct Engine {
    raw: *mut ffi::sx_engine,
}

unsafe impl Send for Engine {}
unsafe impl Sync for Engine {}

/// A configured profile set on the device, owned by its engine.
pub struct ProfileSet<'e> {
    raw: *mut ffi::sx_profiles,
    _engine: std::marker::PhantomData<&'e Engine>,
}

/// A digitised target set on the device, owned by its engine.
pub struct TargetSet<'e> {
    raw: *mut ffi::sx_targets,
    _engine: std::marker::PhantomData<&'e Engine>,
}

impl Engine {
    pub fn new(device: i32) -> Result<Engine> {
        Engine::with_options(ffi::sx_opts { device, ..Default::default() })
    }

    pub fn with_options(opts: ffi::sx_opts) -> Result<Engine> {
        let mut raw = null_mut();
        check(unsafe { ffi::sx_create(&opts, &mut raw) })?;
        Ok(Engine { raw })
    }

    pub fn as_ptr(&self) -> *mut ffi::sx_engine {
        self.raw
    }

    /// `open_hmm` + `HmmReader` + `Hmm::configure` (src/hmmer/parse.rs:42-236,
    /// src/hmmer/model.rs:146-245) in the library: plain or gzip HMMER3 files.
    pub fn load_file(&self, path: &Path) -> Result<ProfileSet<'_>> {
        let c = cstring(&path.to_string_lossy())?;
        let mut raw = null_mut();
        check(unsafe { ffi::sx_profiles_load_file(self.raw, c.as_ptr(), &mut raw) })?;
        Ok(ProfileSet { raw, _engine: std::marker::PhantomData })
    }

    pub fn load_text(&self, text: &str, source: &str) -> Result<ProfileSet<'_>> {
        let src = cstring(source)?;
        let mut raw = null_mut();
        check(unsafe {
            ffi::sx_profiles_load_text(self.raw, text.as_ptr() as *const c_char, text.len(), src.as_ptr(), &mut raw)
        })?;
        Ok(ProfileSet { raw, _engine: std::marker::PhantomData })
    }

    /// Profiles the caller configured itself (the reference's `&[Profile]`),
    /// as plain arrays; the pointers in `arrays` are read during the call only.
    pub fn load_arrays(&self, arrays: &[ffi::sx_profile_arrays]) -> Result<ProfileSet<'_>> {
        let mut raw = null_mut();
        check(unsafe { ffi::sx_profiles_from_arrays(self.raw, arrays.as_ptr(), arrays.len(), &mut raw) })?;
        Ok(ProfileSet { raw, _engine: std::marker::PhantomData })
    }

    /// Digitised targets (codes 0..24, `Targets::dsq` of search.rs:50-80).
    pub fn targets_digital(&self, dsq: &[Vec<u8>]) -> Result<TargetSet<'_>> {
        let mut flat = Vec::with_capacity(dsq.iter().map(|d| d.len()).sum());
        let mut offs = Vec::with_capacity(dsq.len());
        let mut lens = Vec::with_capacity(dsq.len());
        for d in dsq {
            offs.push(flat.len() as i64);
            lens.push(d.len() as i64);
            flat.extend_from_slice(d);
        }
        let mut raw = null_mut();
        check(unsafe {
            ffi::sx_targets_create_digital(self.raw, if flat.is_empty() { null() } else { flat.as_ptr() },
                                           offs.as_ptr(), lens.as_ptr(), lens.len(), &mut raw)
        })?;
        Ok(TargetSet { raw, _engine: std::marker::PhantomData })
    }

    /// The device replacement of `search_profiles` (src/hmmer/search.rs:213-234).
    pub fn search(&self, p: &ProfileSet<'_>, t: &TargetSet<'_>, cfg: &SearchConfig) -> Result<Vec<Hit>> {
        let c = cfg.to_c();
        let mut h = null_mut();
        check(unsafe { ffi::sx_search(self.raw, p.raw, t.raw, &c, &mut h) })?;
        let out = unsafe { take_hits(h) };
        unsafe { ffi::sx_hits_free(h) };
        Ok(out)
    }

    /// Several profile sets against the same targets in one device search;
    /// one hit list per set, each equal to what `search` returns for it.
    pub fn search_many(&self, sets: &[&ProfileSet<'_>], t: &TargetSet<'_>, cfg: &SearchConfig)
        -> Result<Vec<Vec<Hit>>> {
        let c = cfg.to_c();
        let raws: Vec<*const ffi::sx_profiles> = sets.iter().map(|s| s.raw as *const _).collect();
        let mut outs: Vec<*mut ffi::sx_hits> = vec![null_mut(); sets.len()];
        check(unsafe { ffi::sx_search_many(self.raw, raws.as_ptr(), raws.len(), t.raw, &c, outs.as_mut_ptr()) })?;
        let mut all = Vec::with_capacity(outs.len());
        for h in outs {
            all.push(unsafe { take_hits(h) });
            unsafe { ffi::sx_hits_free(h) };
        }
        Ok(all)
    }
}

impl Drop for Engine {
    fn drop(&mut self) {
        unsafe { ffi::sx_destroy(self.raw) }
    }
}

impl ProfileSet<'_> {
    pub fn len(&self) -> usize {
        unsafe { ffi::sx_profiles_count(self.raw) as usize }
    }

    pub fn is_empty(&self) -> bool {
        self.len() == 0
    }

    /// Name and length of profile i (for mapping hits back to models).
    pub fn name_and_len(&self, i: usize) -> Result<(String, usize)> {
        let mut info = std::mem::MaybeUninit::<ffi::sx_profile_info>::zeroed();
        check(unsafe { ffi::sx_profiles_info(self.raw, i as i32, info.as_mut_ptr()) })?;
        let info = unsafe { info.assume_init() };
        let name = unsafe { CStr::from_ptr(info.name) }.to_string_lossy().into_owned();
        Ok((name, info.m as usize))
    }
}

impl Drop for ProfileSet<'_> {
    fn drop(&mut self) {
        unsafe { ffi::sx_profiles_free(self.raw) }
    }
}

impl Drop for TargetSet<'_> {
    fn drop(&mut self) {
        unsafe { ffi::sx_targets_free(self.raw) }
    }
}

unsafe fn slice<'a, T>(p: *const T, n: usize) -> &'a [T] {
    if n == 0 || p.is_null() {
        &[]
    } else {
        std::slice::from_raw_parts(p, n)
    }
}

unsafe fn take_hits(h: *const ffi::sx_hits) -> Vec<Hit> {
    let hs = slice(ffi::sx_hits_array(h), ffi::sx_hits_count(h));
    let ds = slice(ffi::sx_hits_domains(h), ffi::sx_hits_domain_count(h));
    hs.iter()
        .map(|x| {
            let d0 = x.domain_offset as usize;
            Hit {
                profile_index: x.profile_index as usize,
                target_index: x.target_index as usize,
                qlen: x.qlen as usize,
                tlen: x.tlen as usize,
                score: x.score,
                bias: x.bias,
                evalue: x.evalue,
                nexpected: x.nexpected,
                domains: ds[d0..d0 + x.ndomains as usize]
                    .iter()
                    .map(|d| DomainHit {
                        score: d.score,
                        bias: d.bias,
                        c_evalue: d.c_evalue,
                        i_evalue: d.i_evalue,
                        hmm_from: d.hmm_from as usize,
                        hmm_to: d.hmm_to as usize,
                        ali_from: d.ali_from as usize,
                        ali_to: d.ali_to as usize,
                        env_from: d.env_from as usize,
                        env_to: d.env_to as usize,
                        reported: d.reported != 0,
                    })
                    .collect(),
            }
        })
        .collect()
}
