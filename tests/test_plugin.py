"""The C++ plugin surface's rules without a device: accumulation reset on
camera motion, render-target resolution, material conversion, mesh checks."""
import subprocess

from plugin_util import build_test_program


def test_plugin_rules(tmp_path):
    exe = build_test_program(tmp_path)
    r = subprocess.run([exe, "cpu"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    assert "cpu ok" in r.stdout
