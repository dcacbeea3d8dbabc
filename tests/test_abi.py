"""The C ABI without a GPU: struct layouts, exported symbols, constants, and
the error path when no device is present."""
import ctypes as C
import json
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "gargantua.h")


def declared_symbols() -> list[str]:
    names = []
    for path in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if path.endswith(".h"):
            text = open(os.path.join(ROOT, "include", path)).read()
            names += re.findall(r"GG_API\s+[^;(]*?\b(gg_\w+)\s*\(", text)
    return names


def test_library_exports_every_declared_symbol():
    import gargantua_b200 as g

    lib = g.lib()
    names = declared_symbols()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_the_header():
    from gargantua_b200 import _lib

    names = set(declared_symbols())
    assert names <= set(_lib.SIGNATURES) | {n for n in names if n.startswith("gg_server") or n.endswith("_noalloc")}


def test_struct_layouts_match_shadertypes():
    from gargantua_b200 import types as T

    for struct, size in T.LAYOUT.items():
        assert C.sizeof(struct) == size, struct.__name__
    # Offsets ShaderTypes.h produces under Apple simd alignment.
    assert T.MarchUniforms.cameraRight.offset == 16
    assert T.MarchUniforms.cameraForward.offset == 48
    assert T.MarchUniforms.tanHalfFov.offset == 64
    assert T.MarchUniforms.resolution.offset == 72
    assert T.MarchUniforms.tileOrigin.offset == 80
    assert T.MarchUniforms.volumeHalfExtent.offset == 88
    assert T.MarchUniforms.spin.offset == 148
    assert T.MarchUniforms.jitter.offset == 152
    assert T.MarchUniforms.geodesic.offset == 160
    assert T.SplatUniforms.seed.offset == 32
    assert T.Particle.temperature.offset == 24


def test_c_header_compiles_with_layout_asserts(tmp_path):
    """The static assertions in gargantua_types.h hold for a C11 and a C++17
    compiler on this host (the layouts a Swift host sees on Apple)."""
    import subprocess

    src = tmp_path / "t.c"
    src.write_text('#include "gargantua.h"\nint main(void){return (int)sizeof(MarchUniforms) - 192;}\n')
    for cc, std in (("gcc", "-std=c11"), ("g++", "-std=c++17")):
        exe = tmp_path / ("t_" + cc.replace("+", "p"))
        r = subprocess.run(["/usr/bin/" + cc, std, "-x", "c" if cc == "gcc" else "c++", str(src), "-I",
                            os.path.join(ROOT, "include"), "-o", str(exe)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert subprocess.run([str(exe)]).returncode == 0


def test_a_host_shadertypes_header_included_first_is_used(tmp_path):
    """A host that includes its own ShaderTypes.h before gargantua.h keeps
    its structs (the header skips its definitions when the host's include
    guard is set) and the layout pins check the host's structs. The host
    header here is this header's own definitions with one field renamed, so
    the program compiles only if the host's MarchUniforms is the one in
    use."""
    import subprocess

    text = open(os.path.join(ROOT, "include", "gargantua_types.h")).read()
    body = text[text.index("#ifndef GARGANTUA_SHADER_TYPES_H") + len("#ifndef GARGANTUA_SHADER_TYPES_H"):
                text.index("#endif /* GARGANTUA_SHADER_TYPES_H */")]
    assert "float opacityScale;" in body
    host = ("#ifndef GARGANTUA_SHADER_TYPES_H\n#define GARGANTUA_SHADER_TYPES_H\n#include <stdint.h>\n"
            + body.replace("float opacityScale;", "float hostOpacity;") + "\n#endif\n")
    (tmp_path / "ShaderTypes.h").write_text(host)
    src = tmp_path / "host.c"
    src.write_text('#include "ShaderTypes.h"\n#include "gargantua.h"\n'
                   "int main(void) { MarchUniforms u; u.hostOpacity = 0.5f; return (int)sizeof u - 192; }\n")
    exe = tmp_path / "host"
    r = subprocess.run(["/usr/bin/gcc", "-std=c11", str(src), "-I", str(tmp_path), "-I", os.path.join(ROOT, "include"),
                        "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert subprocess.run([str(exe)]).returncode == 0


def test_constants_match_the_reference_table():
    """Every constant in the reference's generated header carries the same
    value in include/gargantua_constants.h (StyleTests.swift:40-44 keeps the
    reference's header equal to its table; this keeps ours equal to theirs)."""
    with open(os.path.join(ROOT, "tests", "golden", "constants.json")) as fh:
        ref = json.load(fh)
    ours = {}
    text = open(os.path.join(ROOT, "include", "gargantua_constants.h")).read()
    for m in re.finditer(r"#define\s+([A-Z0-9_]+)\s+\(([-+0-9.eE]+)[fu]\)", text):
        ours[m.group(1)] = float(m.group(2))
    assert len(ref) == 53
    for symbol, value in ref.items():
        assert symbol in ours, symbol
        assert ours[symbol] == pytest.approx(value, rel=0, abs=0), symbol


def test_every_kernel_loop_names_its_cap():
    """StyleTests.swift:67-75 carried over: every loop in the device sources
    is bounded by a named cap or by a size argument."""
    csrc = os.path.join(ROOT, "gargantua_b200", "csrc")
    for name in os.listdir(csrc):
        if name.endswith((".cu", ".cuh")):
            text = open(os.path.join(csrc, name)).read()
            assert "while (true)" not in text and "for (;;)" not in text, name


def test_context_without_a_device_reports_no_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import gargantua_b200 as g

    with pytest.raises(g.GargantuaError) as e:
        g.Context()
    assert e.value.status == 7  # GG_ERR_NO_DEVICE
    assert "device" in e.value.sentence.lower()


def test_library_structs_match_their_ctypes_mirrors(tmp_path):
    """gg_request, gg_request_result and gg_server_config (this library's own
    structs) have the sizes and offsets the Python mirrors assume."""
    import subprocess

    from gargantua_b200 import types as T

    checks = {
        "gg_request": (T.Request, ["azimuth", "width", "flags", "output", "debug_output", "volume"]),
        "gg_request_result": (T.RequestResult, ["submitted", "ray_steps", "counters", "status"]),
        "gg_server_config": (T.ServerConfig, ["mode", "memory_bytes", "wave_rays", "max_waves_in_flight",
                                             "fp64_policy", "steps_per_round", "refill_idle", "schedule"]),
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gargantua.h"', "int main(void){"]
    for cname, (_, fields) in checks.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "s.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "s"
    r = subprocess.run(["/usr/bin/gcc", "-std=c11", str(src), "-I", os.path.join(ROOT, "include"), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for cname, (struct, fields) in checks.items():
        assert int(got[cname]) == C.sizeof(struct), cname
        for f in fields:
            assert int(got[f"{cname}.{f}"]) == getattr(struct, f).offset, f"{cname}.{f}"


def declared_parameter_counts() -> dict[str, int]:
    """Each GG_API function's parameter count, from its prototype."""
    counts = {}
    for path in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not path.endswith(".h"):
            continue
        text = re.sub(r"/\*.*?\*/", " ", open(os.path.join(ROOT, "include", path)).read(), flags=re.S)
        for name, params in re.findall(r"GG_API\s+[^;(]*?\b(gg_\w+)\s*\(([^)]*)\)\s*;", text):
            params = " ".join(params.split())
            counts[name] = 0 if params in ("", "void") else params.count(",") + 1
    return counts


def test_python_argument_counts_match_the_prototypes():
    """A parameter added on one side only would pass garbage through ctypes."""
    from gargantua_b200 import _lib

    counts = declared_parameter_counts()
    assert len(counts) == len(set(declared_symbols()))
    wrong = {n: (len(args), counts[n]) for n, (_, args) in _lib.SIGNATURES.items()
             if n in counts and len(args) != counts[n]}
    assert not wrong, wrong
    assert set(_lib.SIGNATURES) <= set(counts), set(_lib.SIGNATURES) - set(counts)


def test_swift_module_files_bind_the_header():
    """The Swift system-library module (swift/): its module map's umbrella
    header reaches include/gargantua.h and links the library, and every gg_
    function the sample host calls is declared in the header. (No Swift
    toolchain here compiles it.)"""
    swift = os.path.join(ROOT, "swift")
    modulemap = open(os.path.join(swift, "GargantuaCUDA", "module.modulemap")).read()
    assert 'header "shim.h"' in modulemap and 'link "gargantua_b200"' in modulemap
    shim = open(os.path.join(swift, "GargantuaCUDA", "shim.h")).read()
    target = re.search(r'#include "([^"]*gargantua\.h)"', shim).group(1)
    assert os.path.exists(os.path.normpath(os.path.join(swift, "GargantuaCUDA", target)))
    header = open(os.path.join(ROOT, "include", "gargantua.h")).read()
    declared = set(re.findall(r"GG_API\s+(?:const\s+)?\w+\s*\**\s*(gg_\w+)\(", header))
    called = set(re.findall(r"\b(gg_\w+)\(", open(os.path.join(swift, "Sources", "gg-still", "main.swift")).read()))
    assert called and called <= declared, called - declared
