"""Regenerates tests/golden/reference_kats.json from the reference's own Rust tests.

Run in a container where the reference checkout is mounted (it is not needed
afterwards: the tests read only the committed JSON):

    python tests/golden/extract_kats.py /path/to/Helio

The regular assertions (mip counts, query mips, mip dimensions, occlusion rule,
sphere-vs-plane cases) are parsed from the test sources; the structured ones
(InstanceCullData, select_object_lod, counter decode, work spans, cone rejects,
LOD thresholds, publication budget) are listed here with their file:line.
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

OUT = Path(__file__).resolve().parent / "reference_kats.json"


def grab(path: Path, pattern: str):
    text = path.read_text()
    out = []
    for m in re.finditer(pattern, text):
        line = text[: m.start()].count("\n") + 1
        out.append((m.groups(), line))
    return out


def main(ref: Path) -> None:
    crates = ref / "crates"
    kats: dict = {"source": "t4ce/Helio test sources", "mip_levels": [], "query_mip": [], "mip_dim": [],
                  "occluded": [], "sphere_plane": []}
    for rel in ("helio-pass-hiz/tests/mip_tests.rs", "helio-pass-occlusion-cull/tests/hiz_query_tests.rs"):
        for (w, h, n), line in grab(crates / rel, r"assert_eq!\(mip_levels\((\d+),\s*(\d+)\),\s*(\d+)\)"):
            kats["mip_levels"].append({"w": int(w), "h": int(h), "levels": int(n), "at": f"crates/{rel}:{line}"})
    for rel, fn in (("helio-pass-occlusion-cull/tests/hiz_query_tests.rs", "select_query_mip"),
                    ("helio-pass-occlusion-cull/tests/occlusion_tests.rs", "select_mip")):
        for (w, h, n), line in grab(crates / rel, fn + r"\((\d+),\s*(\d+)\),\s*(\d+)\)"):
            kats["query_mip"].append({"w": int(w), "h": int(h), "mip": int(n), "at": f"crates/{rel}:{line}"})
    rel = "helio-pass-occlusion-cull/tests/occlusion_tests.rs"
    for (b, m, n), line in grab(crates / rel, r"hiz_mip_dim\((\d+),\s*(\d+)\),\s*(\d+)\)"):
        kats["mip_dim"].append({"base": int(b), "mip": int(m), "dim": int(n), "at": f"crates/{rel}:{line}"})
    for (neg, a, b), line in grab(crates / rel, r"assert!\((!?)is_occluded\(([\d.]+),\s*([\d.]+)\)\)"):
        kats["occluded"].append({"near": float(a), "hiz": float(b), "occluded": neg != "!", "at": f"crates/{rel}:{line}"})
    rel = "helio-pass-indirect-dispatch/tests/culling_tests.rs"
    planes = {"NEAR_PLANE": [0, 0, 1, 1], "FAR_PLANE": [0, 0, -1, 100], "LEFT_PLANE": [1, 0, 0, 1],
              "RIGHT_PLANE": [-1, 0, 0, 1], "BOTTOM_PLANE": [0, 1, 0, 1], "TOP_PLANE": [0, -1, 0, 1]}
    vec = r"\[([-\d.]+),\s*([-\d.]+),\s*([-\d.]+)\]"
    for g, line in grab(crates / rel, r"assert!\((!?)sphere_vs_plane\((\w+),\s*" + vec + r",\s*([-\d.]+)\)\)"):
        neg, pl, x, y, z, r = g
        kats["sphere_plane"].append({"planes": [planes[pl]], "center": [float(x), float(y), float(z)],
                                     "radius": float(r), "visible": neg != "!", "at": f"crates/{rel}:{line}"})
    box = [planes[k] for k in ("NEAR_PLANE", "FAR_PLANE", "LEFT_PLANE", "RIGHT_PLANE", "BOTTOM_PLANE", "TOP_PLANE")]
    for g, line in grab(crates / rel, r"assert!\((!?)sphere_in_frustum\(&BOX_FRUSTUM,\s*" + vec + r",\s*([-\d.]+)\)\)"):
        neg, x, y, z, r = g
        kats["sphere_plane"].append({"planes": box, "center": [float(x), float(y), float(z)], "radius": float(r),
                                     "visible": neg != "!", "at": f"crates/{rel}:{line}"})
    # Structured cases, transcribed.
    vg = "crates/helio-pass-virtual-geometry/src/lib.rs"
    kats["instance_cull"] = [
        {"model": [2, 0, 0, 0, 0, 2, 0, 0, 0, 0, 2, 0, 4, 5, 6, 1], "valid": 1, "cone": 1, "max_scale": 2.0,
         "min_scale": 2.0, "at": f"{vg}:315-327"},
        {"model": [4, 0, 0, 0, 0, 2, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1], "valid": 1, "cone": 0, "max_scale": 4.0,
         "min_scale": 1.0, "at": f"{vg}:329-341"},
        {"model": [0] * 16, "valid": 0, "at": f"{vg}:343-348"},
        {"model": ["nan"] + [0] * 15, "valid": 0, "at": f"{vg}:350-357"},
        {"model": [1, 0, 0, 0, 0.5, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1], "cone": 0, "at": f"{vg}:361-365"},
        {"model": [-1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1], "cone": 0, "at": f"{vg}:366-371"},
    ]
    errs = [0.0, 0.01, 0.02, 0.04, 0.08, 0.16, 0.32, 0.64]
    kats["select_lod"] = [
        {"errors": errs, "lod_count": 8, "max_scale": 1.0, "focal": 1000.0, "closest": 100.0, "max_error": 1.0,
         "lod": 4, "at": f"{vg}:377"},
        {"errors": errs, "lod_count": 8, "max_scale": 1.0, "focal": 1000.0, "closest": 10.0, "max_error": 1.0,
         "lod": 1, "at": f"{vg}:378"},
        {"errors": errs, "lod_count": 8, "max_scale": 2.0, "focal": 1000.0, "closest": 100.0, "max_error": 1.0,
         "lod": 3, "at": f"{vg}:379"},
    ]
    kats["counter_decode"] = {"counters": [123, 4, 0, 2, 5, 0, 0, 1, 0, 0, 6], "visible_meshlets": 123,
                              "rejected_meshlets": 4, "visible_objects": 8, "lod_range": [1, 5],
                              "max_available_lod": 6, "short_is_none": 10, "at": f"{vg}:390-403"}
    kats["lod_quality_px"] = {"low": 4.0, "medium": 2.0, "high": 1.0, "ultra": 0.5, "at": f"{vg}:195-202"}
    kats["budget"] = {"default": 262144, "publication_bytes": 9 * 1024 * 1024 + 44,
                      "clamp": [[65536, 65536], [4294967295, 262144]], "at": f"{vg}:301-308"}
    cull = "crates/helio-pass-virtual-geometry/tests/cull_tests.rs"
    kats["cone_reject"] = [
        {"camera": [0, 0, -10], "apex": [0, 0, 0], "axis": [0, 0, 1], "cutoff": 0.5, "reject": True,
         "at": f"{cull}:281-289"},
        {"camera": [0, 0, 10], "apex": [0, 0, 0], "axis": [0, 0, 1], "cutoff": 0.5, "reject": False,
         "at": f"{cull}:291-299"},
        {"camera": [1, 2, 3], "apex": [1, 2, 3], "axis": [0, 0, 1], "cutoff": 0.5, "reject": False,
         "at": f"{cull}:301-308"},
    ]
    kats["farthest_corner"] = {"samples": [0.2, 0.3, 0.9, 0.4], "max": 0.9, "near": 0.8, "occluded": False,
                               "at": f"{cull}:310-315"}
    reb = "crates/helio/src/scene/virtual_geometry/rebuild.rs"
    kats["work_spans"] = {"objects": [[3, 0], [5, 1], [7, 64], [11, 65], [13, 130]],
                          "expected": [[5, 0], [7, 0], [11, 0], [11, 64], [13, 0], [13, 64], [13, 128]],
                          "at": f"{reb}:234-259"}
    # append_unique_meshlets: records 3 -> descriptors with first_index 11, 12 and 7 -> 20,
    # referenced as [3, 3, 7, 3, 7] (the test's helper gives every record one LOD).
    text = (ref / reb).read_text()
    t0 = text.index("fn repeated_instances_share_one_descriptor_copy")
    body = text[t0: text.index("#[test]", t0)]
    ids = dict(re.findall(r"let (\w+) = VirtualMeshId\((\d+)\);", body))
    recs = {ids[n]: [int(x) for x in re.findall(r"meshlet\((\d+)\)", lst)]
            for n, lst in re.findall(r"\((\w+), record\(vec!\[([^\]]*)\]\)\)", body)}
    refs = [int(ids[n]) for n in re.search(r"\[((?:\w+,\s*)+\w+)\],\s*&records", body).group(1).replace(" ", "").split(",")]
    first_idx = [int(x) for x in re.search(r"\.collect::<Vec<_>>\(\),\s*\[([\d,\s]+)\]", body).group(1).split(",")]
    bases = {ids[n]: int(v) for n, v in re.findall(r"assert_eq!\(bases\[&(\w+)\],\s*(\d+)\)", body)}
    line = text[:t0].count("\n") + 1
    kats["unique_meshlets"] = {"meshes": {k: v for k, v in recs.items()}, "references": refs,
                               "expected_first_index": first_idx, "bases": bases,
                               "at": f"{reb}:{line}-{line + body.count(chr(10))}"}
    kats["layout_sizes"] = {"GpuMeshletEntry": 64, "GpuVgObject": 128, "GpuVgDraw": 16, "GpuVgWorkItem": 8,
                            "InstanceCullData": 16, "CullUniforms": 48, "IndirectCullUniforms": 112,
                            "DrawIndexedIndirect": 20, "GpuInstanceData": 144, "GpuCameraUniforms": 368,
                            "at": "crates/libhelio/src/meshlet.rs:131-167; "
                                  "crates/helio-pass-indirect-dispatch/tests/uniforms_tests.rs:37-40,153-158; "
                                  f"{vg}:296-299"}
    bench = "crates/examples/meshlet_cull_benchmark.rs"
    kats["benchmark"] = {"total": 1048576, "cases": [[1, 1048576], [16, 65536], [4096, 256], [65536, 16]],
                         "overflow_probe": {"capacity_delta": 17, "counters": [1048576, 17]},
                         "at": f"{bench}:35,235-240,284-294,368"}
    OUT.write_text(json.dumps(kats, indent=1) + "\n")
    print(f"wrote {OUT}: " + ", ".join(f"{k}={len(v)}" for k, v in kats.items() if isinstance(v, list)))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/extract_kats.py <path of the Helio checkout>")
    main(Path(sys.argv[1]))
