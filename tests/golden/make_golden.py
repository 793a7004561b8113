"""Extract the reference's own known-answer vectors into ``reference_kats.json``.

Run with ``RS_REFERENCE_ROOT`` set to the root of a checkout of the
reference crate (rustfs-erasure-codec 9.1.0).  The reference files are read
as text only: the known-answer literals are copied out of assertions in the
reference test suite, the error enum's variants and messages out of
src/errors.rs, and CodecOptions::default() out of src/core/options.rs; the
file/line of each source is recorded beside it.  Nothing here executes
reference code.

    RS_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import re

REF = os.environ.get("RS_REFERENCE_ROOT", "")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def line_of(text, pos):
    return text.count("\n", 0, pos) + 1


def parse_ints(s):
    s = re.sub(r"//[^\n]*", "", s)
    return [int(t, 0) for t in re.findall(r"0x[0-9a-fA-F]+|\d+", s)]


def bracket_after(text, start):
    """Return (body, end) of the first balanced [...] at or after start."""
    i = text.index("[", start)
    depth = 0
    for j in range(i, len(text)):
        if text[j] == "[":
            depth += 1
        elif text[j] == "]":
            depth -= 1
            if depth == 0:
                return text[i + 1 : j], j
    raise ValueError("unbalanced")


def main():
    if not REF or not os.path.isdir(REF):
        raise SystemExit("set RS_REFERENCE_ROOT to the root of a reference crate checkout")
    kats = {"source": "rustfs-erasure-codec 9.1.0 test suite (literal assertions)"}

    # --- GF(2^8) field (src/galois_8/tests.rs)
    rel = "src/galois_8/tests.rs"
    t = read(rel)
    p = t.index("static BACKBLAZE_LOG_TABLE")
    body, _ = bracket_after(t, t.index("=", p))
    kats["gf8_backblaze_log_table"] = {"where": f"{rel}:{line_of(t, p)}", "values": parse_ints(body)}
    fn = t.index("fn test_galois()")
    fn_end = t.index("\n}\n", fn)
    g = t[fn:fn_end]
    kats["gf8_mul"] = [
        {"a": int(a), "b": int(b), "expect": int(e), "where": f"{rel}:{line_of(t, fn + m.start())}"}
        for m in re.finditer(r"assert_eq!\(mul\((\d+), (\d+)\), (\d+)\)", g)
        for a, b, e in [m.groups()]
    ]
    kats["gf8_exp"] = [
        {"a": int(a), "n": int(n), "expect": int(e), "where": f"{rel}:{line_of(t, fn + m.start())}"}
        for m in re.finditer(r"assert_eq!\(exp\((\d+), (\d+)\), (\d+)\)", g)
        for a, n, e in [m.groups()]
    ]
    inp_pos = g.index("let input = [")
    inp, _ = bracket_after(g, inp_pos)
    # The test replays four slice operations on `output1`; each is followed by
    # the array it must equal.
    ops = []
    for m in re.finditer(r"(mul_slice_xor|mul_slice)\((\d+), &input, &mut output1\);", g):
        kind, coef = m.group(1), int(m.group(2))
        chk = re.compile(r"assert_eq!\((\w+)\[i\], output1\[i\]\)").search(g, m.end())
        exp_pos = g.rfind(f"let {chk.group(1)} = [", 0, chk.start())
        body, _ = bracket_after(g, g.index("=", exp_pos))
        ops.append({"op": kind, "c": coef, "expect": parse_ints(body),
                    "where": f"{rel}:{line_of(t, fn + m.start())}"})
    kats["gf8_slice_ops"] = {"input": parse_ints(inp), "ops": ops}

    # --- classic golden vectors (tests/golden_vectors.rs)
    rel = "tests/golden_vectors.rs"
    t = read(rel)
    gv = {}
    for name in ["golden_encode_4x2_incrementing_input", "golden_reconstruct_data_4x2_incrementing_input",
                 "golden_reconstruct_4x2_incrementing_input", "golden_encode_4x2_seeded_random_input",
                 "golden_encode_4x2_all_zero_input", "golden_encode_4x2_repeated_pattern_input"]:
        p = t.index(f"fn {name}()")
        end = t.index("\n}\n", p)
        body = t[p:end]
        csum = re.search(r"checksum_shards\(&\w+\), (0x[0-9a-f]+)\)", body)
        entry = {"where": f"{rel}:{line_of(t, p)}", "checksum": int(csum.group(1), 16) if csum else None}
        for idx in (4, 5):
            m = re.search(rf"shards\[{idx}\],\s*vec!\[", body)
            if m:
                arr, _ = bracket_after(body, m.end() - 1)
                entry[f"parity{idx}"] = parse_ints(arr)
        gv[name] = entry
    kats["classic_4x2_golden"] = gv
    p = t.index("fn seeded_data")
    kats["classic_4x2_golden"]["seeded_input"] = {"len": 61, "seed": 0xA5A51024,
                                                  "generator": "rand 0.10 SmallRng::seed_from_u64, random::<u8>()",
                                                  "where": f"{rel}:{line_of(t, p)}"}
    p = t.index("fn repeated_pattern_data")
    kats["classic_4x2_golden"]["pattern"] = {"len": 61, "pattern": [0xDE, 0xAD, 0xBE, 0xEF],
                                             "where": f"{rel}:{line_of(t, p)}"}

    # --- classic 2+2 (src/tests/mod.rs test_reconstruct)
    rel = "src/tests/mod.rs"
    t = read(rel)
    p = t.index("fn test_reconstruct()")
    body = t[p: t.index("\n}\n", p)]
    m = re.search(r"let mut shards: \[\[u8; 3\]; 4\] = ", body)
    start, _ = bracket_after(body, m.end() - 1)
    m2 = re.search(r"let expect: \[\[u8; 3\]; 4\] = ", body)
    exp, _ = bracket_after(body, m2.end() - 1)
    kats["classic_2x2"] = {"where": f"{rel}:{line_of(t, p)}", "initial": parse_ints(start),
                           "expect": parse_ints(exp)}

    # --- Leopard GF(2^16) (src/core/leopard_gf16/tests.rs)
    rel = "src/core/leopard_gf16/tests.rs"
    t = read(rel)
    p = t.index("let expected_skew: [u16; 8] =")
    body, _ = bracket_after(t, t.index("=", p))
    kats["lgf16_fft_skew_prefix"] = {"where": f"{rel}:{line_of(t, p)}", "values": parse_ints(body)}
    lp = {}
    for name in ("go_parity0", "go_parity1"):
        p = t.index(f"let {name}: [u8; 16] =")
        body, _ = bracket_after(t, t.index("=", p))
        lp[name] = {"where": f"{rel}:{line_of(t, p)}", "values": parse_ints(body)}
    kats["lgf16_3x2_parity_prefix"] = {"k": 3, "m": 2, "shard_size": 64,
                                       "data": "byte j of shard i = (i*64 + j) & 0xff", **lp}
    p = t.index("let expected: [[u16; 3]; 2] =")
    body, _ = bracket_after(t, t.index("=", p))
    kats["lgf16_3x2_coefficients"] = {"where": f"{rel}:{line_of(t, p)}", "rows": parse_ints(body)}

    # --- Leopard GF(2^8) table invariants (src/core/leopard_gf8/tests.rs)
    rel = "src/core/leopard_gf8/tests.rs"
    t = read(rel)
    p = t.index("assert_eq!(255, tables.log_lut[0]);")
    kats["lgf8_table_invariants"] = {"where": f"{rel}:{line_of(t, p)}", "log_lut0": 255, "exp_lut0": 1}

    # --- encoding-format stable identity (tests/encoding_format_identity.rs)
    rel = "tests/encoding_format_identity.rs"
    t = read(rel)
    for name, key in (("GF8_ID_V1", "format_id_gf8_custom_1x1"), ("TOWER_GF16_ID_V1", "format_id_tower_custom_1x1")):
        p = t.index(f"const {name}: &[u8] =")
        body, _ = bracket_after(t, t.index("=", p))
        kats[key] = {"where": f"{rel}:{line_of(t, p)}", "bytes": parse_ints(body)}
    kats["format_id_gf8_custom_1x1"]["custom_row"] = [0x87]
    kats["format_id_tower_custom_1x1"]["custom_row"] = [[0x12, 0x34]]

    # --- the error enum (src/errors.rs): variants in declaration order (the
    # C ABI returns discriminant + 1) and each variant's as_str message.
    rel = "src/errors.rs"
    t = read(rel)
    p = t.index("pub enum Error {")
    body = t[p + len("pub enum Error {"): t.index("}", p)]
    variants = re.findall(r"^\s*(\w+),", body, flags=re.M)
    q = t.index("fn as_str(self)")
    msgs = {}
    for v in variants:
        m = re.compile(r"Error::%s\s*=>\s*\{?\s*\"([^\"]*)\"" % v).search(t, q)
        msgs[v] = m.group(1)
    kats["error_enum"] = {"where": f"{rel}:{line_of(t, p)}", "variants": variants, "messages": msgs}

    # --- CodecOptions::default() (src/core/options.rs): field -> value
    # (booleans and integers as numbers, enum values by variant name).
    rel = "src/core/options.rs"
    t = read(rel)
    p = t.index("impl Default for CodecOptions")
    body = t[t.index("Self {", p): t.index("}", t.index("Self {", p))]
    defaults = {}
    for name, val in re.findall(r"(\w+):\s*([\w:]+),", body):
        if val in ("true", "false"):
            defaults[name] = int(val == "true")
        elif val.isdigit():
            defaults[name] = int(val)
        else:
            defaults[name] = val.split("::")[-1]
    kats["codec_options_default"] = {"where": f"{rel}:{line_of(t, p)}", "fields": defaults}

    with open(OUT, "w") as f:
        json.dump(kats, f, indent=1, sort_keys=True)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
