"""The C++ host API (include/optixrender.hpp) through the headless
render_json program, which replaces the reference's GL viewer main.cpp."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import optixrender_b200 as rt

CLI = Path(rt.LIBRARY_PATH).parent / "render_json"

SCENE = """{
  "width": 48, "height": 32, "depth": 6, "spp": 4,
  "filter": {"type": "box"},
  "camera": {"look_from": [0.5, 0.5, -1.6], "look_at": [0.5, 0.5, 0.5], "up": [0, 1, 0]},
  "light": [{"type": "quad", "position": [0.375, 0.999, 0.375], "u": [0, 0, 0.25], "v": [0.25, 0, 0],
             "radiance": [17, 12, 4]},
            {"type": "point", "position": [0.5, 0.6, 0.2], "radiance": [0.3, 0.3, 0.3]}],
  "shape": [{"type": "mesh", "mesh_path": "room.obj", "material": "white"},
            {"type": "mesh", "mesh_path": "room.obj", "material": "gold",
             "translate": [0.3, 0, 0.3], "scale": [0.3, 0.3, 0.3]}],
  "material": [{"type": "diffuse", "name": "white", "albedo": [0.73, 0.73, 0.73], "roughness": 0.0},
               {"type": "conductor", "name": "gold", "roughness": 0.3}],
  "integrator": {"rng": "pcg32"}
}"""

ROOM = """v 0 0 0
v 1 0 0
v 1 0 1
v 0 0 1
v 0 1 0
v 1 1 0
v 1 1 1
v 0 1 1
f 1 2 3 4
f 5 8 7 6
f 4 3 7 8
f 1 4 8 5
f 2 6 7 3
"""


def write_scene(d: Path):
    (d / "room.obj").write_text(ROOM)
    (d / "scene.json").write_text(SCENE)
    return d / "scene.json"


def read_ppm(path):
    data = Path(path).read_bytes()
    parts = data.split(b"\n", 3)
    w, h = map(int, parts[1].split())
    return np.frombuffer(parts[3], np.uint8).reshape(h, w, 3)


def test_cli_reports_errors(tmp_path):
    r = subprocess.run([str(CLI), str(tmp_path / "missing.json"), str(tmp_path / "out")], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "error 4" in r.stderr


def test_python_and_json_agree_on_scene_contents(tmp_path):
    s = rt.Scene()
    o, cam = s.load_json(write_scene(tmp_path))
    assert s.counts() == {"triangles": 20, "meshes": 2, "lights": 2, "media": 0}
    assert (o.width, o.height, o.spp, o.rng) == (48, 32, 4, rt.RNG_PCG32)


@pytest.mark.gpu
def test_cli_matches_python_api(tmp_path):
    path = write_scene(tmp_path)
    r = subprocess.run([str(CLI), str(path), str(tmp_path / "out"), "2"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    img = read_ppm(tmp_path / "out.ppm")
    s = rt.Scene()
    o, cam = s.load_json(path)
    o.progressive = 1
    rr = rt.Renderer(s, o)
    rr.set_camera(cam)
    rr.render()
    rr.render()
    px = rr.download_pixels()
    ref = px.view(np.uint8).reshape(px.shape + (4,))[::-1, :, :3]
    assert np.array_equal(img, ref)
    assert img.mean() > 5


def test_facade_compiles_with_textures_and_server(tmp_path):
    """Every wrapper of the C++ facade type-checks against the C ABI."""
    src = tmp_path / "use.cpp"
    src.write_text("""#include "optixrender.hpp"
int main() {
    rt::Scene s;
    int t = s.AddTexture(std::vector<uint8_t>(16, 255), 2, 2);
    rt::Material m(rt::Diffuse);
    m.texture_ids[0] = t;
    rt::Server srv;
    int sid = srv.AddScene(s);
    rt_job_desc j{};
    j.scene = sid;
    int64_t id = srv.Submit(j);
    rt_job_status st = srv.Wait(id, 1000.0);
    std::vector<uint32_t> px(16);
    srv.DownloadPixels(id, px.data());
    srv.Release(id);
    return int(st.state) + int(srv.Stats().jobs_done);
}
""")
    inc = Path(__file__).resolve().parents[1] / "include"
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", str(inc), str(src)], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
