"""The autotuner's search and cache, against a fake context (no GPU)."""
import json

from pulse_b200 import autotune


class FakeCtx:
    """last_render_ms = a cost model of the knobs; stack_depth 16 drops
    pushes, iteration caps of 10 bind."""

    def __init__(self):
        self.ms = 0.0
        self.overflows = 0
        self.cap_hits = 0
        self.calls = 0

    def stats(self):
        return {"last_render_ms": self.ms, "stack_overflows": self.overflows, "iter_cap_hits": self.cap_hits}

    def render(self, p):
        self.calls += 1
        p = dict(autotune.KNOB_DEFAULTS, **p)
        self.ms = 10.0 + abs(p["wf_segments"] - 3) + abs(p["trace_blocks"] - 6) * 0.5 + (32 - p["stack_depth"]) * -0.1
        if p["stack_depth"] < 24:
            self.overflows += 1
        if p["iter_cap"] < 100:
            self.ms -= 0.5
            self.cap_hits += 1


def test_default_space_keeps_the_image():
    """Every knob of the default space renders the same bits; the stack depth
    (which can drop subtrees) is not among them."""
    assert "stack_depth" not in autotune.DEFAULT_SPACE
    assert set(autotune.DEFAULT_SPACE) == {"wf_segments", "trace_blocks", "block_size", "step_policy", "ray_sort"}


def test_tune_picks_fastest(tmp_path):
    ctx = FakeCtx()
    path = tmp_path / "t.json"
    best = autotune.tune(ctx, ctx.render, dict(max_depth=8), "k", path=path)
    assert best["wf_segments"] == 3 and best["trace_blocks"] == 6
    assert best["max_depth"] == 8 and "stack_depth" not in best
    data = json.loads(path.read_text())
    (entry,) = data.values()
    assert entry["best"]["wf_segments"] == 3 and entry["best"]["trace_blocks"] == 6


def test_tune_rejects_traversal_guards(tmp_path):
    """With the stack depth or the iteration cap in an explicit space, a
    candidate whose frames dropped a push or hit a cap is never chosen."""
    ctx = FakeCtx()
    best = autotune.tune(ctx, ctx.render, {}, "k3", space={"stack_depth": [16, 24, 32], "iter_cap": [10, 100000]},
                         path=tmp_path / "g.json")
    assert best["stack_depth"] == 24  # 16 is faster in the model but overflows
    assert best["iter_cap"] == 100000  # 10 is faster in the model but binds
    data = json.loads((tmp_path / "g.json").read_text())
    (entry,) = data.values()
    assert any(row["overflow"] for row in entry["table"])


def test_tune_uses_cache(tmp_path):
    ctx = FakeCtx()
    path = tmp_path / "t.json"
    autotune.tune(ctx, ctx.render, {}, "k", path=path)
    n = ctx.calls
    again = autotune.tune(ctx, ctx.render, {"spp": 2}, "k", path=path)
    assert ctx.calls == n and again["spp"] == 2 and again["wf_segments"] == 3
    autotune.tune(ctx, ctx.render, {}, "k", path=path, force=True)
    assert ctx.calls > n


def test_call_time_overrides_last_render_ms(tmp_path):
    ctx = FakeCtx()

    def call(p):
        ctx.render(p)
        return 100.0 - p["trace_blocks"]  # the caller's own clock prefers more blocks

    best = autotune.tune(ctx, call, {}, "k2", space={"trace_blocks": [2, 4, 8]}, path=tmp_path / "c.json")
    assert best["trace_blocks"] == 8


def test_signature_buckets():
    a = autotune.signature("batched", 36_819_968, 14_037_560, 32, dict(nee_mode=2, max_depth=8))
    b = autotune.signature("batched", 40_000_000, 15_000_000, 32, dict(nee_mode=2, max_depth=8))
    c = autotune.signature("batched", 40_000_000, 15_000_000, 31, dict(nee_mode=2, max_depth=8))
    assert a == b and a != c
