"""Builds tests/plugin/plugin_test.cpp against the C++ plugin surface."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "pulse_b200")
SRC = os.path.join(ROOT, "tests", "plugin", "plugin_test.cpp")


def build_test_program(out_dir) -> str:
    from pulse_b200 import build as pbuild
    pbuild.build()
    pbuild.build_plugin()
    exe = os.path.join(str(out_dir), "plugin_test")
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", SRC, "-o", exe, f"-L{PKG}", "-lpulse_plugin",
                           "-lpulse_cuda", f"-Wl,-rpath,{PKG}"])
    return exe
