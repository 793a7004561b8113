"""The C-ABI library loads on a CPU-only machine and exports every entry point
declared in include/rsgpu.h.  No compute call is made here."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rsgpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rsgpu_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["rsgpu_codec_new", "rsgpu_encode", "rsgpu_reconstruct", "rsgpu_verify",
                 "rsgpu_verify_with_workspace", "rsgpu_encode_batch"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    import rsgpu

    lib = rsgpu.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_reports_version_and_error_text():
    import rsgpu

    lib = rsgpu.lib()
    assert b"sm_100a" in lib.rsgpu_version()
    assert b"zero length" in lib.rsgpu_error_string(11)


def test_codec_without_gpu_fails_loudly():
    import rsgpu

    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(rsgpu.RsError) as e:
        rsgpu.ReedSolomon(10, 4)
    assert e.value.name == "NoDevice"


def test_argument_validation_precedes_device_use():
    # with_options checks run before any device query (src/core/codec.rs:274-297).
    import rsgpu

    with pytest.raises(rsgpu.RsError) as e:
        rsgpu.ReedSolomon(0, 4)
    assert e.value.name == "TooFewDataShards"
    with pytest.raises(rsgpu.RsError) as e:
        rsgpu.ReedSolomon(4, 0)
    assert e.value.name == "TooFewParityShards"
    with pytest.raises(rsgpu.RsError) as e:
        rsgpu.ReedSolomon(200, 57)
    assert e.value.name == "TooManyShards"
