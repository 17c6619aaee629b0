"""The C++ plugin surface on the GPU: the Cornell box driven frame by frame
through the plugin's systems (mesh extraction with U16 and U32 index buffers,
material data, mesh instances, accumulation on a still camera, the path-tracer
node, the upscaling node) gives the same texels, bit for bit, as the
library's Python front end, and the upscaled image equals the resample of the
same target."""
import struct
import subprocess

import numpy as np
import pytest

from plugin_util import build_test_program
from pulse_b200 import scenes
from pulse_b200.tracer import Scene, Target, render_forward

pytestmark = pytest.mark.gpu

W, H, FRAMES, UP = 40, 30, 3, (80, 60)
PARAMS = dict(max_depth=5, nee_mode=2, light_pick=1, quirks=0)


def write_scene(path, desc, moves=(), frames=FRAMES):
    b = bytearray()
    b += struct.pack("<II", desc.params["bins"], desc.params["max_leaf"])
    b += struct.pack("<I", len(desc.meshes))
    for k, m in enumerate(desc.meshes):
        idx = np.asarray(m.indices).astype(np.uint32).ravel()
        kind = 1 if k % 2 == 0 and idx.max() < 65536 else 2  # both index widths
        nv = len(m.positions)
        b += struct.pack("<III", nv, idx.size, kind)
        b += np.asarray(m.positions, np.float32).tobytes()
        b += np.asarray(m.normals, np.float32).tobytes()
        b += np.asarray(m.uvs, np.float32).tobytes()
        b += (idx.astype(np.uint16) if kind == 1 else idx).tobytes()
    b += struct.pack("<I", len(desc.materials))
    for mt in desc.materials:
        b += np.asarray(mt.base_color[:4], np.float32).tobytes() + np.asarray(mt.emissive[:4], np.float32).tobytes()
        b += struct.pack("<fff", mt.perceptual_roughness, mt.reflectance, mt.metallic)
    b += struct.pack("<I", len(desc.instances))
    for inst in desc.instances:
        b += struct.pack("<II", inst.mesh, inst.material) + np.asarray(inst.columns(), np.float32).tobytes()
    b += np.asarray(desc.view.inverse_view_proj, np.float32).tobytes()
    b += np.asarray(desc.view.world_position, np.float32).tobytes()
    b += struct.pack("<III", W, H, frames)
    b += struct.pack("<IIII", PARAMS["nee_mode"], PARAMS["max_depth"], PARAMS["light_pick"], PARAMS["quirks"])
    b += struct.pack("<II", *UP)
    b += struct.pack("<I", len(moves))
    for frame, i, m in moves:
        b += struct.pack("<II", frame, i) + np.asarray(m, np.float32).T.reshape(16).tobytes()
    path.write_bytes(bytes(b))


def test_plugin_frames_match_front_end(ctx, tmp_path):
    desc = scenes.cornell(W, H)
    exe = build_test_program(tmp_path)
    scene_file, out_file = tmp_path / "scene.bin", tmp_path / "out.bin"
    write_scene(scene_file, desc)
    r = subprocess.run([exe, "render", str(scene_file), str(out_file)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert f"accumulation_count {FRAMES - 1}" in r.stdout
    raw = out_file.read_bytes()
    got = np.frombuffer(raw[:W * H * 16], np.float32).reshape(H, W, 4)
    up = np.frombuffer(raw[W * H * 16:], np.uint16).reshape(UP[1], UP[0], 4)
    sc = Scene(ctx)
    p = desc.params
    ids = [sc.upload_mesh(m, p["bins"], p["max_leaf"]) for m in desc.meshes]
    sc.set_materials(desc.materials)
    sc.set_instances(desc.instances, ids)
    tg = Target(ctx, W, H)
    for acc in range(FRAMES):
        render_forward(sc, desc.view, tg, acc, **PARAMS)
    ref = tg.download()
    ref_up = tg.resample(UP[0], UP[1], 0)
    tg.close()
    sc.close()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(up, ref_up.view(np.uint16))


def test_plugin_moving_instances_match_front_end(ctx, tmp_path):
    """Frames in which only transforms change take the plugin's incremental
    path (pulse_instances_update); the accumulated image equals the front end
    rebuilding every instance every frame, as the reference does."""
    desc = scenes.cornell(W, H)
    n = len(desc.instances)
    frames = 4
    base = [np.asarray(inst.object_world, np.float32) for inst in desc.instances]
    moves = [(1, n - 1, scenes.trs(np.array([0.05, 0.0, 0.0]), np.eye(3)) @ base[n - 1]),
             (2, 0, scenes.trs(np.array([0.0, 0.02, 0.0]), np.eye(3)) @ base[0]),
             (2, n - 2, scenes.trs(np.array([-0.04, 0.0, 0.03]), np.eye(3)) @ base[n - 2])]
    exe = build_test_program(tmp_path)
    scene_file, out_file = tmp_path / "scene.bin", tmp_path / "out.bin"
    write_scene(scene_file, desc, moves, frames)
    r = subprocess.run([exe, "render", str(scene_file), str(out_file)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert f"incremental {frames - 1}" in r.stdout, r.stdout
    got = np.frombuffer(out_file.read_bytes()[:W * H * 16], np.float32).reshape(H, W, 4)
    sc = Scene(ctx)
    p = desc.params
    ids = [sc.upload_mesh(m, p["bins"], p["max_leaf"]) for m in desc.meshes]
    sc.set_materials(desc.materials)
    tg = Target(ctx, W, H)
    for k in range(frames):
        for frame, i, m in moves:
            if frame == k:
                desc.instances[i].object_world = m
        sc.set_instances(desc.instances, ids)
        render_forward(sc, desc.view, tg, k, **PARAMS)
    ref = tg.download()
    tg.close()
    sc.close()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_plugin_realtime_gi_matches_front_end(ctx, tmp_path):
    """The realtime plugin (src/pulse): PulseCamera resolution, primary-hit
    G-buffer, PulseNode into the GI target, upscaling node -- equal to the
    front end's gbuffer_primary + render_gi and the target's resample."""
    from pulse_b200.tracer import gbuffer_primary, render_gi
    desc = scenes.cornell(W, H)
    exe = build_test_program(tmp_path)
    scene_file, out_file = tmp_path / "scene.bin", tmp_path / "out.bin"
    write_scene(scene_file, desc, frames=2)
    r = subprocess.run([exe, "gi", str(scene_file), str(out_file)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    raw = out_file.read_bytes()
    got = np.frombuffer(raw[:W * H * 16], np.float32).reshape(H, W, 4)
    up = np.frombuffer(raw[W * H * 16:], np.uint16).reshape(UP[1], UP[0], 4)
    sc = Scene(ctx)
    p = desc.params
    ids = [sc.upload_mesh(m, p["bins"], p["max_leaf"]) for m in desc.meshes]
    sc.set_materials(desc.materials)
    sc.set_instances(desc.instances, ids)
    gb = gbuffer_primary(sc, desc.view, W, H, quirks=PARAMS["quirks"])
    tg = Target(ctx, W, H)
    render_gi(sc, gb, tg, quirks=PARAMS["quirks"])
    ref = tg.download()
    ref_up = tg.resample(UP[0], UP[1], 0)
    tg.close()
    sc.close()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(up, ref_up.view(np.uint16))
