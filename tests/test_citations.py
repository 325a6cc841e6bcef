"""Reference citations: every `<file>.ts:<a>-<b>` (and `.md`) citation in the C ABI header, the
oracle, the package, the tests, the bench and the design notes points inside the cited file of the
reference project, and the citations of the boundary's members point at those members.

The reference project is read from $L3D_REFERENCE (default: the mount point used while this
repository was built); the test is skipped where it is not present.
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("L3D_REFERENCE", "/root/reference")

pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "frontend")),
                                reason="the reference project is not mounted")

CITE = re.compile(r"([A-Za-z0-9_.-]+\.(?:ts|md))((?::\d+(?:-\d+)?)(?:,\d+(?:-\d+)?)*)")

# (file, first cited line) -> text that line of the reference holds: the members the C ABI and
# the Python mirror stand in for
ANCHORS = {
    ("dense-stereo.ts", 11): "interface StereoView",
    ("dense-stereo.ts", 16): "interface SolveOptions",
    ("dense-stereo.ts", 32): "interface CoarseLevel",
    ("dense-stereo.ts", 38): "interface StereoOptions",
    ("dense-stereo.ts", 44): "MAX_SOURCES",
    ("dense-stereo.ts", 46): "GEOMETRIC_WEIGHT",
    ("dense-stereo.ts", 61): "class DenseStereo",
    ("dense-stereo.ts", 80): "constructor(",
    ("dense-stereo.ts", 175): "setImage(",
    ("dense-stereo.ts", 185): "async solve(",
    ("dense-stereo.ts", 242): "get hypotheses()",
    ("dense-stereo.ts", 250): "async filter(",
    ("dense-stereo.ts", 269): "private async sliced(",
    ("dense-stereo.ts", 301): "async filteredMap(",
    ("dense-stereo.ts", 309): "async depthMap(",
    ("dense-stereo.ts", 314): "private params(",
    ("dense-stereo.ts", 333): "Math.imul(ref + 1",
    ("dense-stereo.ts", 357): "destroy()",
    ("tsdf-volume.ts", 13): "class BrickGrid",
    ("tsdf-volume.ts", 67): "interface IntegrationView",
    ("tsdf-volume.ts", 158): "class TsdfVolume",
    ("tsdf-volume.ts", 171): "constructor(",
    ("tsdf-volume.ts", 220): "visibleBricks(",
    ("tsdf-volume.ts", 240): "async integrate(",
    ("tsdf-volume.ts", 270): "async read()",
    ("tsdf-volume.ts", 279): "destroy()",
    ("depth-maps.ts", 9): "function upsampleDepth(",
    ("depth-maps.ts", 66): "function unpackDepthSample(",
    ("camera.ts", 28): "function scaleIntrinsics(",
    ("camera.ts", 73): "function relativePose(",
    ("surface-nets.ts", 47): "function extractSurface(",
    ("point-accumulator.ts", 16): "class PointAccumulator",
    ("gray-image.ts", 12): "function rgbaToGray(",
}


def _reference_files():
    files = {}
    for d, dirs, fs in os.walk(REF):
        dirs[:] = [x for x in dirs if x not in ("node_modules", ".git", ".angular")]
        for f in fs:
            files.setdefault(f, []).append(os.path.join(d, f))
    return files


def _sources():
    out = []
    for d in ("include", "oracle", "luvas.io-3d_b200", "tests"):
        for dd, dirs, fs in os.walk(os.path.join(ROOT, d)):
            dirs[:] = [x for x in dirs if x not in ("_build", "__pycache__", "lib")]
            out += [os.path.join(dd, f) for f in fs if f.endswith((".h", ".cu", ".cpp", ".py"))]
    out += [os.path.join(ROOT, f) for f in ("bench.py", "__graft_entry__.py", "DESIGN.md",
                                            "INTEGRATION.md", "BASELINE.md", "README.md")]
    return [p for p in out if os.path.exists(p)]


def _citations():
    files = _reference_files()
    for path in _sources():
        for ln, line in enumerate(open(path, errors="replace"), 1):
            for m in CITE.finditer(line):
                cands = files.get(m.group(1))
                if not cands or len(cands) != 1:
                    continue  # a file name the reference does not hold once (e.g. README.md)
                for part in m.group(2)[1:].split(","):
                    a, _, b = part.partition("-")
                    yield (os.path.relpath(path, ROOT), ln, m.group(1), cands[0], int(a),
                           int(b or a))


def test_citations_point_inside_the_cited_files():
    lines = {}
    bad = []
    n = 0
    for where, ln, name, path, a, b in _citations():
        n += 1
        if path not in lines:
            lines[path] = sum(1 for _ in open(path, errors="replace"))
        if not (1 <= a <= b <= lines[path]):
            bad.append(f"{where}:{ln}: {name}:{a}-{b} (the file has {lines[path]} lines)")
    assert n > 100
    assert not bad, "\n".join(bad)


def test_member_citations_point_at_the_members():
    text = {}
    bad = []
    for where, ln, name, path, a, b in _citations():
        want = ANCHORS.get((name, a))
        if want is None:
            continue
        if path not in text:
            text[path] = open(path, errors="replace").read().split("\n")
        if want not in text[path][a - 1]:
            bad.append(f"{where}:{ln}: {name}:{a} holds {text[path][a - 1].strip()!r}, not {want!r}")
    assert not bad, "\n".join(bad)
