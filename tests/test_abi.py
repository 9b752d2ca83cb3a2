"""The C ABI library loads without a GPU, exports every symbol declared in
include/galaxy_bh.h, and its host-side checks reject bad input before any
device work."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "galaxy_bh.h")).read()
    return sorted(set(re.findall(r"\b(galaxy_bh_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from galaxy_b200 import _lib, build
    build.build()
    return _lib.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared_symbols()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    from galaxy_b200 import _lib
    assert set(_lib.SIGNATURES) == set(names)


def test_abi_version(lib):
    assert lib.galaxy_bh_abi_version() == 1


def test_record_sizes_match_header():
    from galaxy_b200 import _lib
    assert _lib.EVOLVE_STATE_DTYPE.itemsize == 32
    assert _lib.GPU_CELL_DTYPE.itemsize == 64
    assert _lib.GPU_ENTRY_DTYPE.itemsize == 16
    assert _lib.BH_SETTINGS_DTYPE.itemsize == 32


def test_canonical_fixture_through_host_dtypes():
    """The frozen records, packed with the engine's host dtypes, give the
    reference's 144-byte fixture (nbody_gpu.rs:1453-1489)."""
    import json
    from galaxy_b200 import _lib
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_vectors.json")))
    f = g["canonical_fixture_fields"]
    s = np.zeros((), _lib.BH_SETTINGS_DTYPE)
    s["info"], s["physics"] = f["settings"]["info"], f["settings"]["physics"]
    b = np.zeros((), _lib.GPU_BODY_DTYPE)
    b["position_mass"], b["meta"] = f["body"]["position_mass"], f["body"]["meta"]
    e = np.zeros((), _lib.GPU_ENTRY_DTYPE)
    e["data"] = f["entry"]["data"]
    c = np.zeros((), _lib.GPU_CELL_DTYPE)
    for k in ("center_half_mass", "com", "range_depth", "children"):
        c[k] = f["cell"][k]
    raw = s.tobytes() + b.tobytes() + e.tobytes() + c.tobytes()
    assert raw.hex() == g["canonical_fixture_hex"]


def test_no_device_is_reported_cleanly(lib):
    """Without a GPU, opening a device fails with BH_NO_DEVICE and a message."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from galaxy_b200 import NbodyGpu, EngineUnavailable
    with pytest.raises(EngineUnavailable, match="CUDA"):
        NbodyGpu()


def test_null_and_bad_arguments_rejected(lib):
    from galaxy_b200 import _lib
    assert lib.galaxy_bh_device_open(0, None) == _lib.BH_INVALID_ARG
    cfg = _lib.BhConfig(0.5, 0.01, 1.0, 0, 16, 0, 0)  # bucket 0
    out = C.c_uint64()
    rc = lib.galaxy_bh_batch_footprint(None, C.byref(cfg), 1, C.byref(out))
    assert rc == _lib.BH_INVALID_ARG


def test_footprint_grows_with_bodies(lib):
    from galaxy_b200 import _lib
    cfg = _lib.BhConfig(0.5, 0.01, 1.0, 1, 48, 0, 0)
    sizes = []
    for n in (1 << 10, 1 << 16, 1 << 20):
        counts = np.array([n], np.uint32)
        out = C.c_uint64()
        assert lib.galaxy_bh_batch_footprint(_lib.ptr(counts), C.byref(cfg), 1, C.byref(out)) == 0
        sizes.append(out.value)
    assert sizes[0] < sizes[1] < sizes[2]
    # bucket 1, depth 16: <= 9 cells per body; ~216 B per cell (records, node
    # groups of four child slots, f64 aggregates, links) + ~100 B per body
    assert sizes[2] < 2200 * (1 << 20)


def test_host_state_validation():
    from galaxy_b200.nbody_gpu import bodies_to_state, Config
    b = np.zeros((4, 5))
    b[:, 4] = 1.0
    b[2, 0] = np.nan
    with pytest.raises(ValueError, match="body 2"):
        bodies_to_state(b)
    b[2, 0] = 1e300
    with pytest.raises(ValueError, match="finite f32"):
        bodies_to_state(b)
    with pytest.raises(ValueError, match="at least|2..="):
        bodies_to_state(np.zeros((1, 5)) + 1)
    with pytest.raises(ValueError, match="bucket"):
        Config(bucket=0).validate()


def _arity(params: str) -> int:
    params = params.strip()
    if params in ("", "void"):
        return 0
    return len([x for x in params.split(",") if x.strip()])


def header_declarations() -> dict:
    """name -> parameter count of every function declared in the header."""
    text = open(os.path.join(ROOT, "include", "galaxy_bh.h")).read()
    return {m[0]: _arity(m[1]) for m in re.findall(
        r"\b(?:int|uint32_t|size_t)\s+(galaxy_bh_\w+)\s*\(([^)]*)\)\s*;", text)}


def test_rust_crate_binds_the_whole_header():
    """The Rust crate (galaxy_b200/rust) declares every function of the
    header with the same parameter count, so a maintainer wiring the
    reference's runtime binds the whole surface."""
    decl = header_declarations()
    assert set(decl) == set(declared_symbols())
    src = open(os.path.join(ROOT, "galaxy_b200", "rust", "src", "lib.rs")).read()
    rust = {m[0]: _arity(m[1]) for m in re.findall(r"pub fn (galaxy_bh_\w+)\(([^)]*)\)", src)}
    assert set(rust) == set(decl), sorted(set(rust) ^ set(decl))
    for name, n in decl.items():
        assert rust[name] == n, (name, rust[name], n)
