"""The C-ABI library loads on a CPU-only machine and exports every entry point
declared in include/rsgpu.h.  No compute call is made here."""
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


@pytest.mark.parametrize("k,m,family,mode,want", [
    # explicit families: src/core/leopard.rs:225-237 (ceil(k / m') * m' <= order - m', m' = next_pow2(m))
    (192, 64, "leopard_gf8", "disabled", "leopard_gf8"),
    (193, 63, "leopard_gf8", "disabled", "TooManyShards"),   # total 256, but 4 x 64 > 256 - 64
    (200, 100, "leopard_gf8", "disabled", "TooManyShards"),  # total above 256
    (32768, 16384, "leopard_gf16", "disabled", "leopard_gf16"),
    (49153, 16383, "leopard_gf16", "disabled", "TooManyShards"),
    (40000, 30000, "leopard_gf16", "disabled", "TooManyShards"),
    # automatic selection from Classic: src/core/leopard.rs:191-223
    (300, 100, "classic", "disabled", "TooManyShards"),
    (300, 100, "classic", "as_needed", "leopard_gf16"),
    (200, 56, "classic", "as_needed", "classic"),
    (10, 4, "classic", "prefer_gf16", "leopard_gf16"),
    (100, 128, "classic", "prefer_leopard", "leopard_gf8"),
    (100, 130, "classic", "prefer_leopard", "leopard_gf16"),  # parity above 128
])
def test_leopard_family_resolution_and_limits(k, m, family, mode, want):
    # Family resolution and shape validation run on the host before any
    # device query: without a GPU an accepted shape reaches the device query
    # (NoDevice), a rejected one fails first.  With a GPU the resolved family
    # is read back.
    import rsgpu

    opts = rsgpu.CodecOptions(codec_family=family, leopard_mode=mode)
    try:
        codec = rsgpu.ReedSolomon(k, m, opts)
    except rsgpu.RsError as e:
        if e.name == "NoDevice":
            assert want in ("classic", "leopard_gf8", "leopard_gf16"), (k, m, family, mode)
            return
        assert e.name == want, (k, m, family, mode)
        return
    assert codec.codec_family() == want, (k, m, family, mode)


# C struct (include/rsgpu.h) -> its ctypes mirror in the Python package.
STRUCT_MIRRORS = {
    "rsgpu_options": "_Options", "rsgpu_cache_stats": "CacheStats", "rsgpu_stream_options": "StreamOptions",
    "rsgpu_stream_status": "StreamStatus", "rsgpu_mix_op": "MixOp", "rsgpu_plan": "Plan",
    "rsgpu_mix_options": "MixOptions", "rsgpu_mix_info": "MixInfo", "rsgpu_tune_options": "TuneOptions",
    "rsgpu_tune_sample": "TuneSample", "rsgpu_train_options": "TrainOptions",
    "rsgpu_server_options": "ServerOptions", "rsgpu_request": "Request", "rsgpu_completion": "Completion",
    "rsgpu_server_stats": "ServerStats",
}


def c_members(name):
    """Member names of `typedef struct name { ... } name;` in the header."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, flags=re.S).group(1)
    out = []
    for decl in body.split(";"):
        for i, part in enumerate(decl.split(",")):
            ids = re.findall(r"[A-Za-z_]\w*", re.sub(r"\[[^\]]*\]", "", part))
            if ids:
                out.append(ids[-1])
    return out


def test_every_header_struct_has_a_mirror():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    assert sorted(re.findall(r"typedef struct (rsgpu_\w+) \{", text)) == sorted(STRUCT_MIRRORS)


def test_ctypes_mirrors_match_the_header_layout(tmp_path):
    # The Python mirror passes these structs by pointer; a size or offset that
    # differs from the C declaration corrupts memory silently.
    import shutil
    import subprocess

    import rsgpu

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    checks, want = [], []
    for cname, pyname in STRUCT_MIRRORS.items():
        cls = getattr(rsgpu, pyname)
        checks.append(f'printf("%zu\\n", sizeof({cname}));')
        want.append(ctypes_sizeof(cls))
        members = set(c_members(cname))
        for field, _ in cls._fields_:
            if field in members:
                checks.append(f'printf("%zu\\n", offsetof({cname}, {field}));')
                want.append(getattr(cls, field).offset)
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "rsgpu.h"\nint main(void) {\n'
                   + "\n".join(checks) + "\nreturn 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == want, [(c, g, w) for c, g, w in zip(checks, got, want) if g != w]


def ctypes_sizeof(cls):
    import ctypes

    return ctypes.sizeof(cls)


def header_param_counts():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for name, params in re.findall(r"\b(rsgpu_\w+)\s*\(([^;{}]*?)\)\s*;", text):
        params = params.strip()
        out[name] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_ctypes_signatures_match_the_header_parameter_counts():
    # The Python mirror binds every entry point the header declares, each
    # with as many arguments as the header gives it.
    import rsgpu

    lib = rsgpu.lib()
    for name, n in header_param_counts().items():
        argtypes = getattr(lib, name).argtypes
        assert argtypes is not None, f"{name} is not bound"
        assert len(argtypes) == n, (name, len(argtypes), n)
