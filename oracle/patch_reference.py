"""Prepare the azimuth sources for the oracle build (test infrastructure).

Copies ``src/`` of the reference checkout into ``oracle/_ref/src`` (git-ignored)
and applies mechanical edits.  None of them changes what the code computes:

1. GCC rejects azimuth's MSVC-only duplicate member names inside anonymous
   unions (src/azimuth_math.h:88-300 vec types, src/azimuth_entity.h:81-85,
   src/azimuth_light.h:15-37).  Every repeated name is an alias of the same
   offset, so the repeats are renamed; all uses still resolve to the first
   declaration at that offset.
2. ``Random01`` (src/azimuth_math.cpp:1-8) returns the shared counter-based RNG
   instead of libc ``rand()``.
3. ``GetSampleCoord`` (src/azimuth_main.cpp:1135) announces the pixel and
   sample to the RNG; ``TraceRay`` (src/azimuth_main.cpp:966) opens one RNG
   node per activation; ``ComputeSampleWeight`` (src/azimuth_main.cpp:1208)
   hands the finished sample's colour to the harness, which records it when
   asked for per-sample radiance.  Each is one inserted line.
4. ``src/azimuth_platform.h`` selects the platform layer with ``#if _WIN32``;
   the oracle selects the POSIX stand-in in ``oracle/shim`` instead, and the
   Win32 platform files are not copied.

Usage: python oracle/patch_reference.py <reference src dir> <output dir>
"""
import os
import re
import shutil
import sys

SKIP = {"azimuth_platform_win32.cpp", "azimuth_platform_win32.h"}
DECL = re.compile(r"^(\s*[A-Za-z_][\w\s\*]*?[\s\*])([A-Za-z_]\w*)(\s*\[[^\]]*\])?(\s*;.*)$")


def rename_union_duplicates(text):
    """Rename repeated member names among the structs of each anonymous union."""
    lines = text.split("\n")
    out = []
    depth = 0
    union_depths = []          # brace depth at which each open union's body lives
    seen = []                  # names declared so far in each open union
    dup_count = 0
    for line in lines:
        code = line.split("//")[0]
        opens = code.count("{")
        closes = code.count("}")
        if re.match(r"^\s*union\s*\{", code):
            union_depths.append(depth + 1)
            seen.append(set())
        elif union_depths and depth == union_depths[-1] + 1 and opens == 0 and closes == 0:
            m = DECL.match(line)
            if m and "(" not in code:
                name = m.group(2)
                if name in seen[-1]:
                    dup_count += 1
                    line = m.group(1) + name + "_AzAlias%d" % dup_count + (m.group(3) or "") + m.group(4)
                else:
                    seen[-1].add(name)
        depth += opens - closes
        while union_depths and depth < union_depths[-1]:
            union_depths.pop()
            seen.pop()
        out.append(line)
    return "\n".join(out), dup_count


def replace_once(text, old, new, what):
    n = text.count(old)
    if n != 1:
        raise SystemExit("patch_reference: expected one '%s' anchor, found %d" % (what, n))
    return text.replace(old, new)


def regex_once(text, pattern, repl, what):
    new, n = re.subn(pattern, repl, text, count=1, flags=re.S)
    if n != 1:
        raise SystemExit("patch_reference: anchor for %s not found" % what)
    return new


def main(src, dst):
    os.makedirs(dst, exist_ok=True)
    for name in sorted(os.listdir(src)):
        if name in SKIP or not (name.endswith(".h") or name.endswith(".cpp")):
            continue
        with open(os.path.join(src, name), encoding="latin-1") as f:
            text = f.read()
        if name in ("azimuth_math.h", "azimuth_entity.h", "azimuth_light.h"):
            text, n = rename_union_duplicates(text)
            if n == 0:
                raise SystemExit("patch_reference: no duplicate members found in " + name)
        if name == "azimuth_math.cpp":
            text = replace_once(text, "Result = ((f32)rand())/RAND_MAX;",
                                "Result = AzOracleRandom01();", "Random01 body")
        if name == "azimuth_main.cpp":
            text = regex_once(
                text,
                r"(\nGetSampleCoord\(u32 SampleX, u32 SampleY, u32 Row, u32 Col,\s*f32 OneOverSampleCountSqrt\)\{\n)",
                r"\1    AzOracleBeginSample(Row, Col, SampleX, SampleY);\n", "GetSampleCoord")
            text = regex_once(
                text,
                r"(\nTraceRay\(scene \*Scene, ray3 Ray, u32 RecursionDepth,[^{;]*\)\{\n)",
                r"\1    AZ_ORACLE_NODE_SCOPE();\n", "TraceRay")
            text = regex_once(
                text,
                r"(\nComputeSampleWeight\(vec3 Color, vec2 SampleCoord, pixel \*Pixels,[^{;]*\)\{\n)",
                r"\1    AzOracleSampleDone(Color.x, Color.y, Color.z);\n", "ComputeSampleWeight")
        if name == "azimuth_platform.h":
            if text.count("#if _WIN32") != 2:
                raise SystemExit("patch_reference: platform selector changed")
            text = text.replace("#if _WIN32", "#if 1")
        with open(os.path.join(dst, name), "w", encoding="latin-1") as f:
            f.write(text)
    return 0


if __name__ == "__main__":
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    sys.exit(main(sys.argv[1], sys.argv[2]))
