"""The C++ oracle under AddressSanitizer and UndefinedBehaviorSanitizer: the
oracle built with -fsanitize=address,undefined (no recovery) runs BVH builds
(including the degenerate and empty cases), instance preparation, ray queries,
every estimator with quirks on and off, the FP64 converged mean, the realtime
GI pass and the FP64 adjoint on small scenes, in a child process with the
sanitizer runtime preloaded.  Any report fails the child."""
import os
import subprocess
import sys
import textwrap

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = textwrap.dedent("""
    import sys
    from pathlib import Path
    sys.path.insert(0, {root!r})
    import numpy as np
    import oracle
    oracle.LIB = Path({lib!r})
    from pulse_b200 import scenes
    rng = np.random.default_rng(3)
    for n, bins, leaf in [(1, 2, 1), (9, 16, 8), (257, 20, 8), (1000, 32, 4)]:
        c = rng.normal(size=(n, 1, 3)) * 4
        v = (c + rng.normal(size=(n, 3, 3)) * 0.3).astype(np.float32)
        prims = np.zeros((n, 12), np.float32)
        for k in range(3):
            prims[:, 4 * k:4 * k + 3] = v[:, k]
        oracle.build_blas(prims, bins, leaf)
    try:
        oracle.build_blas(np.zeros((20, 12), np.float32), 16, 1)  # every centroid equal
    except Exception:
        pass
    oracle.build_tlas(np.zeros((0, 9), np.float32))
    d = scenes.cornell(24, 20)
    sb = oracle.assemble(d.meshes, d.materials, d.instances, 16, 4)
    rays = oracle.primary_rays(d.view, 24, 20)
    oracle.trace(sb, rays, nthreads=2)
    for mode in (0, 1, 2):
        for quirks in (1, 0):
            oracle.render(sb, d.view, 24, 20, 0, nthreads=2, max_depth=4, nee_mode=mode, quirks=quirks,
                          light_pick=mode == 2)
    oracle.render_mean64(sb, d.view, 24, 20, 2, pixels=np.arange(0, 480, 7), nthreads=2, max_depth=4, nee_mode=2)
    gb = oracle.gbuffer_primary(sb, d.view, 24, 20)
    oracle.render_gi(sb, gb, 12, 10, nthreads=2, spp=2, max_depth=3)
    dl = np.ones((20, 24, 4), np.float32)
    oracle.backward(sb, d.view, 24, 20, 2, dl, nthreads=2, max_depth=4, nee_mode=2, light_pick=1, quirks=0)
    s = scenes.spheres_1080p(level=2, n_instances=6, width=16, height=12)
    sb2 = oracle.assemble_desc(s)
    oracle.render(sb2, s.view, 16, 12, 0, nthreads=2, max_depth=3, nee_mode=2, light_pick=1, quirks=0)
    print("sanitized oracle ok")
""")


def _runtime(name):
    p = subprocess.run(["g++", f"-print-file-name={name}"], capture_output=True, text=True).stdout.strip()
    return p if os.path.isabs(p) and os.path.exists(p) else None


@pytest.mark.timeout(600)
def test_oracle_under_asan_and_ubsan(tmp_path):
    asan = _runtime("libasan.so")
    if asan is None:
        pytest.skip("no AddressSanitizer runtime")
    lib = tmp_path / "liboracle_asan.so"
    flags = [f for f in oracle.CXXFLAGS if f != "-O2"] + ["-O1", "-g", "-fno-omit-frame-pointer",
                                                          "-fsanitize=address,undefined",
                                                          "-fno-sanitize-recover=all"]
    subprocess.check_call(["g++", *flags, "-o", str(lib), str(oracle.SRC)])
    env = dict(os.environ, LD_PRELOAD=asan, ASAN_OPTIONS="detect_leaks=0:abort_on_error=0:exitcode=23",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1:exitcode=24")
    r = subprocess.run([sys.executable, "-c", DRIVER.format(root=ROOT, lib=str(lib))], capture_output=True,
                       text=True, env=env, timeout=540)
    assert r.returncode == 0 and "sanitized oracle ok" in r.stdout, (r.returncode, r.stdout[-2000:],
                                                                     r.stderr[-4000:])
