"""Every C-ABI entry point either waits for the pipelined frames in flight
(pulse_ctx_set_pipeline) before it touches the device, or is one of the
calls that need not: pure host calls, creation of new objects, the
asynchronous download (which waits for its target's last frame through
events) and the render, which decides per call.  A new entry point that
forgets the wait would read, write or free memory a running frame uses; this
check reads the source, so it runs without a GPU.
"""
import os
import re

SRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pulse_b200", "csrc", "api.cu")
HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "pulse_cuda.h")

# Entry points that do not wait for the frames in flight, and why.
NO_WAIT = {
    "pulse_default_params": "host only",
    "pulse_default_gi_params": "host only",
    "pulse_last_error": "host only",
    "pulse_debug_fail_allocations": "host only",
    "pulse_scene_counts": "host only",
    "pulse_target_device_ptr": "returns a pointer; consumers order themselves through pulse_ctx_get_stream",
    "pulse_ctx_create": "a new context has no frames",
    "pulse_scene_create": "a new scene has no buffers",
    "pulse_target_create": "a new target is read by no frame",
    "pulse_target_download_async": "its copy waits for the target's last frame (event)",
    "pulse_target_download_wait": "waits on the host for the copy, which follows the frame",
}
# Entry points that delegate to render_impl, which waits unless the frame itself is pipelined.
VIA_RENDER = {"pulse_render_forward", "pulse_render_count"}


def _bodies():
    src = open(SRC).read()
    out = {}
    for m in re.finditer(r"^(?:int32_t|void|const char\*) (pulse_\w+)\(", src, re.M):
        start = src.index("{", m.end())
        depth, i = 0, start
        while True:
            if src[i] == "{":
                depth += 1
            elif src[i] == "}":
                depth -= 1
                if depth == 0:
                    break
            i += 1
        out[m.group(1)] = src[start:i]
    return out, src


def test_every_entry_point_waits_for_frames_in_flight():
    bodies, src = _bodies()
    declared = set(re.findall(r"PULSE_API [\w\s\*]+?\b(pulse_\w+)\(", open(HEADER).read()))
    assert declared <= set(bodies), declared - set(bodies)
    for name in declared:
        body = bodies[name]
        if name in NO_WAIT:
            continue
        if name in VIA_RENDER:
            assert "render_impl(" in body, name
            continue
        assert "quiesce(" in body, f"{name} does not wait for the pipelined frames in flight"
    # render_impl waits whenever the frame is not pipelined
    impl = src[src.index("static int32_t render_impl("):]
    impl = impl[:impl.index("\n}\n")]
    assert "if (!piped) quiesce(ctx);" in impl
    # the double-buffered instance update waits on its in-place path
    assert "if (!fast) quiesce(ctx);" in bodies["pulse_instances_set"]
