"""A bounded rendering case for profiler captures.

Renders the spheres benchmark scene (2.59M triangles, resident scene and BVH
of ~0.3 GB, larger than the 126 MB L2) at a reduced frame size and sample
count, so that a capture of a few kernel launches ends in seconds:

  python -m optixrender_b200.profile_case --width 480 --height 270 --spp 2 --frames 2
"""
from __future__ import annotations

import argparse
import sys


def main(argv=None) -> int:
    p = argparse.ArgumentParser()
    p.add_argument("--scene", default="spheres")
    p.add_argument("--width", type=int, default=480)
    p.add_argument("--height", type=int, default=270)
    p.add_argument("--spp", type=int, default=2)
    p.add_argument("--frames", type=int, default=2)
    p.add_argument("--stats", type=int, default=0)
    p.add_argument("--wave-paths", type=int, default=0, help="path slots per wave (0 = the library's choice)")
    a = p.parse_args(argv)
    from . import scenes
    spec = scenes.SCENES[a.scene](width=a.width, height=a.height, spp=a.spp)
    s, r = scenes.build_renderer(spec, collect_stats=a.stats, wave_paths=a.wave_paths)
    for _ in range(a.frames):
        r.render()
    r.synchronize()
    st = r.stats()
    print({k: st[k] for k in ("paths", "extend_rays", "shadow_rays", "launches", "ms_total", "wave_paths")})
    return 0


if __name__ == "__main__":
    sys.exit(main())
