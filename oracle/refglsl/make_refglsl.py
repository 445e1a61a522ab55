"""oracle/refglsl/make_refglsl.py -- TEST INFRASTRUCTURE ONLY.

Writes C++-compilable copies of the reference's compute shaders (every .glsl and
.comp file under the reference's src/Shaders) into a build folder (oracle/_ref/glsl,
git-ignored; nothing of the reference is committed). The copies are compiled
with glsl_shim.h by oracle/Makefile into oracle/_ref/librefglsl.so, a second
oracle that runs the reference's own shader code on the host.

The rewrites are mechanical and change no arithmetic or control flow:
  1. `#version` / `#extension` lines are blanked (not C preprocessor directives).
  2. `__cplusplus` is renamed: the reference guards GLSL-only helpers with
     `#ifndef __cplusplus` (core/primitive_cpp.glsl), which a GLSL compiler never
     defines, so the copy must keep them.
  3. `layout(...) buffer|uniform Name { members };` blocks become their members:
     runtime-sized arrays `T name[];` become bounds-checked views
     (`GLSL_SSBO(T, name)`), other members static variables.
     `layout(...) uniform <image/sampler> name[...];` becomes a static variable and
     `layout(local_size...) in;` is dropped (the C++ host program dispatches the invocations).
  4. Parameter qualifiers: `in T x` -> `T x`, `out T x` / `inout T x` -> `T& x`.
  5. Unsuffixed floating-point literals get an `f` suffix: a GLSL literal such as
     `10e-6` is a float, a C++ one a double.
  6. `void main()` -> `void glsl_main()`.
  7. A non-void function whose body can fall off its end (lighting.glsl
     evalSphereLight when the light is out of range) returns a value-initialised
     (zero) result there; SPIR-V leaves that value undefined, and the restatement
     and the CUDA kernels use zero.
  8. The body of bvh/bvhCollision.glsl's tlas_collide, the closest-hit half of the
     two-level variant (USE_TRAVERSE_TLAS), becomes a call to
     refglsl_unreachable() and a zero return: it names a ClosestHit member (nid)
     and a type and function (Hit, HitBox) that the reference does not define
     (HitBox and Hit exist only commented out, core/collision.glsl:175-195), so no
     compiler accepts it. The any-hit half, tlas_collide_fast, is kept as is and
     never calls it; a driver compiled with USE_TRAVERSE_TLAS defines
     refglsl_unreachable to flag an error should it ever run.

Usage: python make_refglsl.py --ref <reference>/src/Shaders --out <dir>/Shaders
"""
from __future__ import annotations

import argparse
import re
from pathlib import Path

FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")
BLOCK = re.compile(r"layout\s*\([^)]*\)\s*((?:\w+\s+)*?)(uniform|buffer)\s+(\w+)\s*\{([^{}]*)\}\s*(\w*)\s*;", re.S)
OPAQUE = re.compile(r"layout\s*\([^)]*\)\s*uniform\s+(?:(?:readonly|writeonly|coherent|restrict|volatile)\s+)*"
                    r"(\w+)\s+(\w+)\s*(\[[^\]]*\])?\s*;")
LOCAL_SIZE = re.compile(r"layout\s*\([^)]*\)\s*in\s*;")
PARAM = re.compile(r"([(,]\s*)(const\s+)?(inout|out|in)\s+(\w+)(\s+)(\w+)")
FUNC_HEAD = re.compile(r"(\w+)\s+(\w+)\s*\(([^()]*)\)\s*$")
KEYWORDS = {"return", "else", "struct", "if", "while", "for", "switch", "case", "do"}


def _lines(s: str) -> str:
    return "\n" * s.count("\n")


def _block(m: re.Match) -> str:
    out = []
    for decl in m.group(4).split(";"):
        d = " ".join(decl.split())
        if not d:
            continue
        a = re.fullmatch(r"(\w+)\s+(\w+)\s*\[\s*\]", d)
        out.append(f"GLSL_SSBO({a.group(1)}, {a.group(2)})" if a else f"static {d};")
    return " ".join(out) + _lines(m.group(0))


def _param(m: re.Match) -> str:
    lead, const, q, ty, sp, name = m.groups()
    if q == "in":
        return f"{lead}{const or ''}{ty}{sp}{name}"
    return f"{lead}{ty}&{sp}{name}"


def _code_mask(src: str) -> list[bool]:
    """True for characters that are code (not a comment, not a preprocessor line)."""
    mask = [True] * len(src)
    i, n, bol = 0, len(src), True
    while i < n:
        c = src[i]
        if bol and c == "#" or (bol and c in " \t" and src[i:].lstrip(" \t").startswith("#")):
            j = i
            while j < n:
                if src[j] == "\n" and (j == 0 or src[j - 1] != "\\"):
                    break
                j += 1
            for k in range(i, j):
                mask[k] = False
            i = j
            continue
        if src.startswith("//", i):
            j = src.find("\n", i)
            j = n if j < 0 else j
            for k in range(i, j):
                mask[k] = False
            i = j
            continue
        if src.startswith("/*", i):
            j = src.find("*/", i + 2)
            j = n if j < 0 else j + 2
            for k in range(i, j):
                mask[k] = False
            i = j
            continue
        bol = c == "\n"
        i += 1
    return mask


def _add_fallthrough_returns(src: str) -> str:
    mask = _code_mask(src)
    code = "".join(ch if m else (ch if ch == "\n" else " ") for ch, m in zip(src, mask))
    inserts = []
    depth, last_end, open_at, ret_type = 0, 0, -1, None
    for i, ch in enumerate(code):
        if ch == "{":
            if depth == 0:
                head = FUNC_HEAD.search(code[last_end:i])
                ret_type = None
                if head and head.group(1) not in KEYWORDS and head.group(1) != "void":
                    ret_type = head.group(1)
                open_at = i
            depth += 1
        elif ch == "}":
            depth -= 1
            if depth == 0:
                if ret_type:
                    inserts.append((i, f" return {ret_type}(); "))
                ret_type = None
                last_end = i + 1
        elif ch == ";" and depth == 0:
            last_end = i + 1
    for pos, text in reversed(inserts):
        src = src[:pos] + text + src[pos:]
    return src


# rewrite 8: functions whose bodies become a stub, per file
STUBS = {"bvh/bvhCollision.glsl": {"tlas_collide": "{ refglsl_unreachable(); return 0u; }"}}


def _stub_functions(src: str, stubs: dict) -> str:
    mask = _code_mask(src)
    for name, body in stubs.items():
        m = re.search(rf"\b{name}\s*\([^()]*\)\s*\{{", src)
        if not m or not mask[m.start()]:
            raise SystemExit(f"make_refglsl: function {name} not found")
        start = m.end() - 1
        depth = 0
        for i in range(start, len(src)):
            if not mask[i]:
                continue
            if src[i] == "{":
                depth += 1
            elif src[i] == "}":
                depth -= 1
                if depth == 0:
                    src = src[:start] + body + _lines(src[start:i + 1]) + src[i + 1:]
                    break
        mask = _code_mask(src)
    return src


def transform(src: str) -> str:
    src = re.sub(r"^[ \t]*#[ \t]*(version|extension)\b[^\n]*", "", src, flags=re.M)
    src = src.replace("__cplusplus", "TIM_REFGLSL_GLSL_ONLY_GUARD")
    src = BLOCK.sub(_block, src)
    src = OPAQUE.sub(lambda m: f"static {m.group(1)} {m.group(2)}{m.group(3) or ''};", src)
    src = LOCAL_SIZE.sub("", src)
    src = PARAM.sub(_param, src)
    src = PARAM.sub(_param, src)          # overlapping matches (", out a, out b")
    src = FLOAT_LIT.sub(lambda m: m.group(1) + "f", src)
    src = re.sub(r"\bvoid\s+main\s*\(\s*\)", "void glsl_main()", src)
    src = _add_fallthrough_returns(src)
    return src


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference's src/Shaders folder (read only)")
    ap.add_argument("--out", required=True, help="output folder (mirrors the Shaders tree)")
    a = ap.parse_args()
    ref, out = Path(a.ref), Path(a.out)
    n = 0
    for p in sorted(list(ref.rglob("*.glsl")) + list(ref.rglob("*.comp"))):
        dst = out / p.relative_to(ref)
        dst.parent.mkdir(parents=True, exist_ok=True)
        text = transform(p.read_text(encoding="utf-8", errors="replace"))
        rel = p.relative_to(ref).as_posix()
        if rel in STUBS:
            text = _stub_functions(text, STUBS[rel])
        if not dst.exists() or dst.read_text() != text:
            dst.write_text(text)
        n += 1
    print(f"make_refglsl: {n} shader files -> {out}")


if __name__ == "__main__":
    main()
