"""Phase clock of the certifier's warp loop (a measurement build).

Builds the library a second time with ``-DP2C_ENGINE_PROFILE`` into
``_build_profile/`` (beside the product build, which stays untouched): lane 0
of every warp then adds the SM clock cycles of each phase of the engine's loop
(fetch, donation, pool take, idle wait, distance sample, classify, record,
move to the next node, export, finalise, budget check) to a per-file device
array that ``p2c_engine_profile_<file>`` reads back.  Each phase boundary
synchronises the warp, so absolute cycles are inflated by a few hundred per
phase; shares are what the breakdown is for.

Run: ``python -m p2cccd_b200.engine_profile`` (needs a GPU) prints one JSON
line per workload: the plain 20,000-query batch, the two-sphere scene's
certification and two cloth-on-sphere scenes certified in full.
"""
from __future__ import annotations

import ctypes
import json
from pathlib import Path

PHASES = ["fetch", "donate", "pool", "idle", "distance", "classify", "record", "move", "export", "finalise",
          "budget"]
PROFILE_LIB = Path(__file__).resolve().parent.parent / "_build_profile" / "libp2c_b200_profile.so"


def build_profile_library() -> Path:
    from . import build

    return build.build(extra_flags=["-DP2C_ENGINE_PROFILE"], lib=PROFILE_LIB, build_dir=PROFILE_LIB.parent / "obj")


def _read(lib, which: str) -> list[int]:
    out = (ctypes.c_ulonglong * 16)()
    fn = getattr(lib, "p2c_engine_profile_" + which)
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int]
    if fn(ctypes.addressof(out), 1) != 0:
        raise RuntimeError("reading the engine phase clock failed")
    return list(out)[:12]


def _line(tag: str, prof: list[int], ms: float, extra: dict) -> str:
    total = sum(prof[:11])
    iters = max(prof[11], 1)
    return json.dumps({"workload": tag, "ms": ms, **extra, "busy_warp_iterations": prof[11],
                       "share": {n: round(prof[i] / max(total, 1), 4) for i, n in enumerate(PHASES)},
                       "cycles_per_busy_warp_iteration": {n: round(prof[i] / iters, 1) for i, n in enumerate(PHASES)}})


def main() -> None:
    lib_path = build_profile_library()
    from . import _lib

    _lib.LIB_PATH = lib_path  # this process only: every entry point below runs the measurement build
    lib = _lib.load()
    import torch

    from . import certify, scenes, workloads
    from .scene import ScenePipeline

    dev = torch.device("cuda:0")
    cfg = certify.CertConfig(1e-6, 1e-6, 32)
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    w = workloads.plain_queries(workloads.PlainSpec())
    pt, ee = certify.records_to_device(w["vf"], dev), certify.records_to_device(w["ee"], dev)
    ws = certify.Workspace(dev)
    for _ in range(3):
        certify.certify_batch2(pt, ee, 0.0, 1.0, cfg, workspace=ws)
    torch.cuda.synchronize()
    _read(lib, "certify")
    e0, e1 = ev()
    e0.record()
    certify.certify_batch2(pt, ee, 0.0, 1.0, cfg, workspace=ws)
    e1.record()
    torch.cuda.synchronize()
    st = ws.stats()
    print(_line("plain 20,000 queries", _read(lib, "certify"), e0.elapsed_time(e1),
                {"nodes": int(st["nodes_evaluated"]), "max_warp_iterations": int(st["max_warp_iterations"])}),
          flush=True)
    cases = [("two spheres, 2 x 40,960 triangles", scenes.two_spheres(), True),
             ("cloth 129 x 129 on a 12,000-triangle sphere", scenes.cloth_on_sphere(n=129, sphere_lon=60,
                                                                                    sphere_rings=50), False),
             ("cloth 257 x 257 on a 25,000-triangle sphere", scenes.cloth_on_sphere(n=257, sphere_lon=125,
                                                                                    sphere_rings=100), False)]
    for tag, s, excl in cases:
        p = ScenePipeline(s, dev, exclude_self=excl, config=cfg)
        p.step_checked()
        p.fit_capacities()
        summ = p.step_checked()
        p.candidates()
        torch.cuda.synchronize()
        _read(lib, "scene")
        e0, e1 = ev()
        e0.record()
        p.certify()
        e1.record()
        torch.cuda.synchronize()
        print(_line(tag, _read(lib, "scene"), e0.elapsed_time(e1),
                    {"queries": summ["vf_certified"] + summ["ee_certified"]}), flush=True)


if __name__ == "__main__":
    main()
