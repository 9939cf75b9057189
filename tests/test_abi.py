"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares; host-only entry points behave like the reference."""
import ctypes as C
import glob
import os
import re

import pytest

import psift

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(psift_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(psift.LIB_PATH)
    declared = _declared()
    assert len(declared) >= 10
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(_declared()) == set(psift.exported_symbols())


def test_default_config_matches_reference():
    lib = psift.load_library()
    c = psift.CSiftConfig()
    lib.psift_sift_config_default(C.byref(c))
    assert (c.octaves, c.scales, c.upsample_first_octave, c.descriptor_kind, c.max_features) == (3, 3, 1, 0, 4096)
    assert abs(c.contrast_threshold - 0.015) < 1e-9


@pytest.mark.parametrize("kw,msg", [
    (dict(octaves=0), "Invalid `octaves`=0: must be between 1 and 8"),
    (dict(octaves=9), "Invalid `octaves`=9: must be between 1 and 8"),
    (dict(scales=2), "Invalid `scales`=2: must be between 3 and 10 for 3D extrema extraction"),
    (dict(scales=11), "Invalid `scales`=11: must be between 3 and 10 for 3D extrema extraction"),
    (dict(contrast_threshold=0.0), "must be finite and in (0.0, 1.0]"),
    (dict(contrast_threshold=1.5), "must be finite and in (0.0, 1.0]"),
    (dict(contrast_threshold=float("nan")), "must be finite and in (0.0, 1.0]"),
    (dict(contrast_threshold=float("inf")), "must be finite and in (0.0, 1.0]"),
])
def test_config_validation_messages(kw, msg):
    # SiftConfig::validate, src/pipeline.rs:80-103; pinned by tests/pipeline_tests.rs:1335-1363
    cfg = psift.SiftConfig(**kw)
    with pytest.raises(ValueError) as ei:
        psift.Sift.new(cfg)
    assert msg in str(ei.value)


def test_valid_configs_accepted():
    for o in (1, 8):
        for s in (3, 10):
            psift.SiftConfig(octaves=o, scales=s, contrast_threshold=1.0).validate()


@pytest.mark.parametrize("ratio", [0.0, -1.0, 1.5, float("nan"), float("inf")])
def test_invalid_match_ratio_rejected(ratio):
    # Matcher::new, src/pipeline.rs:156-164
    with pytest.raises(ValueError) as ei:
        psift.Matcher.new(psift.MatchOptions(ratio=ratio))
    assert "must be finite and in (0.0, 1.0]" in str(ei.value)


def test_valid_match_options():
    psift.Matcher.new(psift.MatchOptions(ratio=1.0))
    psift.Matcher.new(psift.MatchOptions(ratio=0.01, mutual=True, precision=psift.PRECISION_FP32))
