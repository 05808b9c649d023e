"""The C-ABI boundary without a GPU.

* libnricp_b200.so loads and exports every function include/nricp_b200.h
  declares;
* the ctypes mirrors of the header's structs have the C layout (sizes and
  field offsets from a probe compiled with gcc against the header);
* host-side validation raises the reference's errors before any device work:
  ValueError with the reference's messages for bad meshes, settings, masks and
  landmarks (src/core/mesh.cpp:90-116, src/core/constraints.cpp:8-58), and
  ValueError for an unknown route (bindings.cpp:1527-1531).
"""

from __future__ import annotations

import ctypes as C
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from nricp_b200 import _abi
from nricp_b200 import synthetic as S

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "nricp_b200.h"


def declared_functions() -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(nricp_\w+)\s*\(", text)))


def test_library_exports_every_declared_function():
    from nricp_b200._lib import load

    lib = load()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


STRUCTS = {
    "NricpLevelSettings": _abi.LevelSettings,
    "NricpSolveDesc": _abi.SolveDesc,
    "NricpResult": _abi.Result,
    "NricpProgress": _abi.Progress,
    "NricpTickRecord": _abi.TickRecord,
    "NricpInspect": _abi.Inspect,
    "NricpServerConfig": _abi.ServerConfig,
    "NricpServerStats": _abi.ServerStats,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc for the layout probe")
def test_ctypes_structs_match_the_c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"',
             "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("return 0; }")
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    layout = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True,
                               text=True).stdout.splitlines():
        cname, field, value = line.split()
        layout[(cname, field)] = int(value)
    for cname, cls in STRUCTS.items():
        assert C.sizeof(cls) == layout[(cname, "size")], cname
        for field, _ in cls._fields_:
            assert getattr(cls, field).offset == layout[(cname, field)], (cname, field)


def _case():
    return S.small_case(seed=1)


def test_invalid_meshes_raise_the_reference_messages(dp):
    case = _case()
    bad = case.template_points.copy()
    bad[5, 1] = np.nan
    with pytest.raises(ValueError, match="vertex 5 is not finite"):
        dp.solve_route_b(bad, case.template_faces, case.target_points, case.target_faces,
                         case.level_settings, **case.options)
    faces = case.target_faces.copy()
    faces[2, 1] = len(case.target_points) + 3
    with pytest.raises(ValueError, match="face 2 corner 1 index"):
        dp.solve_route_b(case.template_points, case.template_faces, case.target_points, faces,
                         case.level_settings, **case.options)


def test_invalid_masks_and_landmarks_raise(dp):
    case = _case()
    v = len(case.template_points)
    with pytest.raises(ValueError, match="mask excludes every vertex"):
        dp.solve_route_b(*case.args(), mask=np.zeros(v, bool), **case.options)
    with pytest.raises(ValueError, match="invalid landmarks"):
        dp.solve_route_b(*case.args(), landmark_indices=np.array([1, 1]),
                         landmark_targets=np.zeros((2, 3)), **case.options)
    with pytest.raises(ValueError, match=f"but the template has {v} vertices"):
        dp.solve_route_b(*case.args(), landmark_indices=np.array([v + 4]),
                         landmark_targets=np.zeros((1, 3)), **case.options)


def test_validation_messages_match_the_reference(dp, reference):
    """Same inputs, same ValueError text as the reference's own validation."""
    case = _case()
    bad = case.template_points.copy()
    bad[5, 1] = np.inf
    with pytest.raises(ValueError) as theirs:
        reference.solve(bad, case.template_faces, case.target_points, case.target_faces,
                        case.level_settings, **case.options)
    with pytest.raises(ValueError) as mine:
        dp.solve_route_b(bad, case.template_faces, case.target_points, case.target_faces,
                         case.level_settings, **case.options)
    assert str(mine.value) == str(theirs.value)


def test_unknown_route_is_a_value_error(dp):
    case = _case()
    with pytest.raises(ValueError, match="route"):
        dp.RouteBSession(*case.args(), route="route_z", **case.options)


def test_template_graph_rejects_bad_meshes(dp):
    points, faces = S.icosphere(1)
    faces = faces.copy()
    faces[0, 0] = -1
    with pytest.raises(ValueError, match="out of range"):
        dp.build_template_graph(points, faces)


def test_plan_follows_the_reference_level_sizes(dp):
    # node count per level: min(lround(nodes_initial * growth^level), V)
    # (src/core/graph.cpp:52-58)
    case = S.small_case(seed=2, levels=3, nodes_initial=40)
    desc = _abi.Desc(*case.args(), route=0, **case.options)
    v = len(case.template_points)
    assert dp._plan(desc) == [min(40, v), min(80, v), min(160, v)]


def test_report_serialisation_is_the_references_text(dp):
    """The reference's own report of a route-A run (tests/golden), written
    again from its parsed values, comes out byte for byte (report.cpp:44-106)."""
    import json
    from pathlib import Path

    text = str(np.load(Path(__file__).parent / "golden" / "route_a_small.npz")["out_report"])
    r = json.loads(text)
    nan = lambda d: {k: (float("nan") if v is None else v) for k, v in d.items()}  # noqa: E731
    again = dp.serialize_report(r["route"], r["precision"], r["setup_seconds"], r["solve_seconds"],
                                nan(r["energy"]), nan(r["correspondence"]), [nan(x) for x in r["levels"]],
                                nan(r["settings"]))
    assert again == text


def test_report_non_finite_values_are_null(dp):
    import json

    zero = {k: 0 for k in ("total", "accepted", "rejected_distance", "rejected_normal", "rejected_slope",
                           "rejected_masked", "distance_mean", "distance_p95", "distance_max")}
    text = dp.serialize_report("route_b", "float", 0.0, 0.0,
                               {"point_to_point": float("nan"), "point_to_plane": 0.0, "smoothness": 0.0,
                                "anchor": 0.0, "landmark": float("inf")}, zero, [], {})
    report = json.loads(text)
    assert report["energy"]["point_to_point"] is None and report["energy"]["total"] is None
    assert report["levels"] == [] and report["settings"] == {} and '"levels": [],' in text


def test_device_info_without_a_device(dp):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    info = dp.device_info()
    assert info["available"] is False and info["device"]


@pytest.mark.parametrize("name", ["solve_route_a", "energy_blocks", "assemble_normal_equations",
                                  "solve_normal_equations", "fused_system"])
def test_entry_points_not_provided_say_why(name):
    """The reference module's FP64 CPU route and its CPU teaching interface
    are not part of this device module: reaching one names the reason."""
    import nricp_dp

    with pytest.raises(AttributeError, match="is not provided by this module"):
        getattr(nricp_dp, name)
    assert not hasattr(nricp_dp, name)
