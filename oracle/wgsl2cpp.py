#!/usr/bin/env python3
"""Translate the reference's WGSL compute shaders into C++ so they run on the CPU.

TEST INFRASTRUCTURE ONLY (part of the oracle).  This is how the oracle is
pinned to the reference itself: the shaders of the hot path are read from the
reference checkout at build time, preprocessed exactly as the reference's
``setup_state`` does (``src/gpu_setup.rs:683-709``: the ``//_feat_*`` text
switches and workgroup-size substitution), translated statement by statement
into C++ and compiled next to ``oracle/ref_driver.cpp``.  The generated code
goes only to ``oracle/_ref/`` (git-ignored) — no reference source is stored in
this repository.

Translation rules (the WGSL subset used by these shaders):
  * ``struct`` / ``fn`` / ``let`` / ``var`` / ``for`` / ``if`` map to C++;
    ``var`` without initializer is zero-initialized (WGSL semantics).
  * Float literals become binary32 literals; ``i32()/u32()/f32()`` casts and
    the builtins (exp, atan2, sin, cos, sqrt, ceil, round, max) map to
    binary32 helpers (round = round-half-to-even, as WGSL specifies).
  * A statement ``acc += a * b;`` becomes ``acc = fmaf(a, b, acc);`` — the
    contraction a shader compiler performs; nothing else is fused (the C++ is
    compiled with -ffp-contract=off).
  * Storage/uniform/push-constant bindings become namespace-scope variables
    the driver sets; atomics become plain sequential increments (the driver
    dispatches invocations serially in row-major order); storage arrays are
    bounds-checked (WGSL robust buffer access: reads outside the buffer give
    zero, writes outside it are dropped).

Usage: wgsl2cpp.py <reference_root> <out_dir>
"""
import os
import re
import sys

SHADERS = {
    # name: (relative path, feature switches applied)
    "preprocess_rows": "src/shaders/preprocess_rows.wgsl",
    "preprocess_cols": "src/shaders/preprocess_cols.wgsl",
    "max_rows": "src/shaders/max_rows.wgsl",
    "extract_max": "src/shaders/extract_max.wgsl",
    "walk": "src/shaders/walk.wgsl",
    "characterize": "src/shaders/characterize.wgsl",
    "separable_log": "src/shaders/log_style/separable_log.wgsl",
    "logspace_max": "src/shaders/log_style/logspace_max.wgsl",
    # frame std (StdArray, src/utils.rs:297-640) and the adaptive background filter
    "sum_image_outplace": "src/shaders/sum_image_outplace.wgsl",
    "sum_image_inplace": "src/shaders/sum_image_inplace.wgsl",
    "last_reduction": "src/shaders/last_reduction.wgsl",
    "std_image": "src/shaders/std_image.wgsl",
    "adaptive_filter": "src/shaders/adaptive_filter.wgsl",
    # illumination correction (src/execute_gpu.rs:138-166, 849-884)
    "smooth_mean_frame": "src/shaders/correct_illumination/smooth_mean_frame.wgsl",
    "correct_illumination": "src/shaders/correct_illumination/correct_illumination.wgsl",
}

TYPE_MAP = {
    "i32": "int32_t",
    "u32": "uint32_t",
    "f32": "float",
    "bool": "bool",
    "atomic<u32>": "uint32_t",
    "atomic<i32>": "int32_t",
    "vec2<f32>": "vec2f",
    "vec2<i32>": "ivec2",
    "vec3<u32>": "uvec3",
}


def ctype(t):
    t = t.strip()
    if t in TYPE_MAP:
        return TYPE_MAP[t]
    m = re.fullmatch(r"array<(.+)>", t)
    if m:
        # storage arrays keep WGSL's robust buffer access: out-of-range reads
        # return zero, out-of-range writes are dropped
        return "RobustArray<%s>" % ctype(m.group(1))
    return t  # user struct


def split_comment(line):
    i = line.find("//")
    if i < 0:
        return line, ""
    return line[:i], line[i:]


FLOAT_LIT = re.compile(r"(?<![\w.])(\d+\.\d*|\.\d+)(?![\w.])")


def fix_literals(s):
    return FLOAT_LIT.sub(lambda m: m.group(1) + "f", s)


def top_level_split(expr, op):
    """Split expr at top-level occurrences of the single-char operator op."""
    parts, depth, cur = [], 0, ""
    for ch in expr:
        if ch in "([":
            depth += 1
        elif ch in ")]":
            depth -= 1
        if ch == op and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    parts.append(cur)
    return parts


def has_top_level(expr, ops):
    depth = 0
    for ch in expr:
        if ch in "([":
            depth += 1
        elif ch in ")]":
            depth -= 1
        elif depth == 0 and ch in ops:
            return True
    return False


def translate_expr(e):
    e = fix_literals(e)
    e = re.sub(r"\bbitcast<u32>\s*\(", "wgsl_bitcast_u32(", e)
    e = re.sub(r"\bbitcast<f32>\s*\(", "wgsl_bitcast_f32(", e)
    e = re.sub(r"\bvec2<i32>\s*\(", "ivec2(", e)
    e = re.sub(r"\bvec2<f32>\s*\(", "vec2f(", e)
    e = re.sub(r"\bvec2\s*\(", "vec2f(", e)
    for name in ("i32", "u32", "f32"):
        e = re.sub(r"\b%s\s*\(" % name, "wgsl_%s(" % name, e)
    for b in ("exp", "sqrt", "atan2", "sin", "cos", "ceil", "round", "max", "min", "abs", "floor"):
        e = re.sub(r"(?<![\w.])%s\s*\(" % b, "wgsl_%s(" % b, e)
    e = re.sub(r"\batomicAdd\s*\(", "wgsl_atomicAdd(", e)
    e = re.sub(r"\batomicSub\s*\(", "wgsl_atomicSub(", e)
    return e


def translate_params(plist):
    out = []
    for p in [x.strip() for x in top_level_split(plist, ",") if x.strip()]:
        p = re.sub(r"@builtin\([^)]*\)\s*", "", p)
        name, t = p.split(":", 1)
        out.append("%s %s" % (ctype(t), name.strip()))
    return ", ".join(out)


def translate_statement(code):
    """Translate one line of code (comment already removed)."""
    s = code
    stripped = s.strip()
    if not stripped:
        return s
    indent = s[: len(s) - len(s.lstrip())]

    # fn declarations
    m = re.match(r"fn\s+(\w+)\s*\((.*)\)\s*(->\s*([\w<>]+))?\s*\{\s*$", stripped)
    if m:
        name = m.group(1)
        if name == "main":
            name = "main_"
        ret = ctype(m.group(4)) if m.group(4) else "void"
        return "%sstatic %s %s(%s) {" % (indent, ret, name, translate_params(m.group(2)))

    # for (var i: T = a; cond; step)
    m = re.match(r"for\s*\(\s*var\s+(\w+)\s*:\s*([\w<>]+)\s*=\s*(.*?);(.*);(.*)\)\s*\{\s*$", stripped)
    if m:
        return "%sfor (%s %s = %s;%s;%s) {" % (
            indent, ctype(m.group(2)), m.group(1), translate_expr(m.group(3)),
            translate_expr(m.group(4)), translate_expr(m.group(5)))
    m = re.match(r"for\s*\(\s*var\s+(\w+)\s*=\s*(.*?);(.*);(.*)\)\s*\{\s*$", stripped)
    if m:
        return "%sfor (auto %s = %s;%s;%s) {" % (
            indent, m.group(1), translate_expr(m.group(2)), translate_expr(m.group(3)),
            translate_expr(m.group(4)))

    # if / else if without mandatory parentheses
    m = re.match(r"(\}?\s*(?:else\s+)?)if\s+(.*?)\s*\{\s*$", stripped)
    if m:
        return "%s%sif (%s) {" % (indent, m.group(1), translate_expr(m.group(2)))

    # let / var declarations
    m = re.match(r"let\s+(\w+)\s*:\s*([\w<>]+)\s*=\s*(.*);\s*$", stripped)
    if m:
        return "%sconst %s %s = %s;" % (indent, ctype(m.group(2)), m.group(1), translate_expr(m.group(3)))
    m = re.match(r"let\s+(\w+)\s*=\s*(.*);\s*$", stripped)
    if m:
        return "%sconst auto %s = %s;" % (indent, m.group(1), translate_expr(m.group(2)))
    m = re.match(r"var\s+(\w+)\s*:\s*([\w<>]+)\s*=\s*(.*);\s*$", stripped)
    if m:
        return "%s%s %s = %s;" % (indent, ctype(m.group(2)), m.group(1), translate_expr(m.group(3)))
    m = re.match(r"var\s+(\w+)\s*:\s*([\w<>]+)\s*;\s*$", stripped)
    if m:
        return "%s%s %s{};" % (indent, ctype(m.group(2)), m.group(1))
    m = re.match(r"var\s+(\w+)\s*=\s*(.*);\s*$", stripped)
    if m:
        return "%sauto %s = %s;" % (indent, m.group(1), translate_expr(m.group(2)))

    # acc += a * b;  ->  fused multiply-add
    m = re.match(r"([\w.\[\]]+)\s*\+=\s*(.*);\s*$", stripped)
    if m:
        lhs, rhs = m.group(1), m.group(2)
        if not has_top_level(rhs, "+-/"):
            factors = top_level_split(rhs, "*")
            if len(factors) == 2:
                a, b = (translate_expr(f.strip()) for f in factors)
                lhs_t = translate_expr(lhs)
                return "%s%s = wgsl_fma(%s, %s, %s);" % (indent, lhs_t, a, b, lhs_t)
        return "%s%s += %s;" % (indent, translate_expr(lhs), translate_expr(rhs))

    return indent + translate_expr(stripped)


def translate_struct_field(line):
    code, _ = split_comment(line)
    code = code.strip().rstrip(",")
    if not code:
        return None
    name, t = code.split(":", 1)
    return "    %s %s;" % (ctype(t), name.strip())


def translate(src):
    lines = src.split("\n")
    out = []
    i = 0
    pending_binding = False
    while i < len(lines):
        raw = lines[i]
        code, comment = split_comment(raw)
        st = code.strip()
        if re.match(r"struct\s+\w+\s*\{", st):
            name = re.match(r"struct\s+(\w+)", st).group(1)
            out.append("struct %s {" % name)
            rest = st[st.index("{") + 1:]
            fields_src = []
            if "}" in rest:
                fields_src.append(rest[: rest.index("}")])
            else:
                i += 1
                while "}" not in split_comment(lines[i])[0]:
                    fields_src.append(lines[i])
                    i += 1
                fields_src.append(split_comment(lines[i])[0].split("}")[0])
            for fs in fields_src:
                for part in split_comment(fs)[0].split(","):
                    f = translate_struct_field(part)
                    if f:
                        out.append(f)
            out.append("};")
            i += 1
            continue
        if st.startswith("@group") or st.startswith("@compute"):
            # attribute lines: drop (binding numbers are the driver's business)
            rest = re.sub(r"@\w+(\([^)]*\))?", "", st).strip()
            if rest.startswith("fn"):
                out.append(translate_statement(rest))
            i += 1
            continue
        m = re.match(r"var<([^>]*)>\s*(\w+)\s*:\s*(.*);", st)
        if m:
            out.append("static %s %s{};" % (ctype(m.group(3)), m.group(2)))
            i += 1
            continue
        if not st:
            out.append(comment)
            i += 1
            continue
        out.append(translate_statement(code.rstrip()) + ("  " + comment if comment else ""))
        i += 1
    return "\n".join(out)


def preprocess(src, header, truncate, char_points, log_style):
    # src/gpu_setup.rs:683-709
    s = header + src
    if char_points:
        s = s.replace("//_feat_characterize_points ", "")
    if truncate:
        s = s.replace("//_feat_truncate_preprocessed ", "")
    if log_style:
        s = s.replace("//_feat_LoG ", "")
    s = s.replace("@workgroup_size(_)", "")
    s = s.replace("_workgroup1d_", "256u")
    return s


def main():
    ref, out = sys.argv[1], sys.argv[2]
    os.makedirs(out, exist_ok=True)
    header = open(os.path.join(ref, "src/shaders/params.wgsl")).read() + "\n"
    variants = []
    for name, rel in SHADERS.items():
        src = open(os.path.join(ref, rel)).read()
        if name == "preprocess_cols":
            variants.append((name + "_trunc", preprocess(src, header, True, False, False)))
            variants.append((name + "_notrunc", preprocess(src, header, False, False, False)))
        elif name == "characterize":
            variants.append((name, preprocess(src, header, True, False, False)))
            variants.append((name + "_points", preprocess(src, header, True, True, False)))
        else:
            variants.append((name, preprocess(src, header, True, False, False)))
    for vname, text in variants:
        cpp = translate(text)
        with open(os.path.join(out, "gen_%s.inc" % vname), "w") as f:
            f.write("// generated by oracle/wgsl2cpp.py from the reference's WGSL; do not commit\n")
            f.write("namespace sh_%s {\n%s\n}  // namespace sh_%s\n" % (vname, cpp, vname))
    print("wrote %d shader translations to %s" % (len(variants), out))


if __name__ == "__main__":
    main()
