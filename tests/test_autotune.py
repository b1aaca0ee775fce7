"""The size-class table of alpha-beta launch shapes (sbd_b200/autotune.py):
classes, loading, and applying a class's shape to a context (a stand-in
object here; the shapes themselves are checked on the GPU in
tests/test_gpu_batch.py)."""
import json
import os
import tempfile

from sbd_b200 import autotune


class FakeCtx:
    def __init__(self, na, nb, norb, fits=True):
        self.na, self.nb, self.norb = na, nb, norb
        self.fits = fits
        self.shape = None

    def set_tuning(self, g, t):
        if not self.fits:
            raise RuntimeError("does not fit")
        self.shape = (g, t)


def test_size_classes():
    assert autotune.size_class(200, 200, 10) == "nb<=256,P<=64"
    assert autotune.size_class(2000, 257, 20) == "nb<=512,P<=256"
    assert autotune.size_class(12000, 12000, 36) == "nb<=16384,P<=1024"
    assert autotune.size_class(3, 70000, 64) == f"nb<={1 << 62},P<=4096"  # P = 2080


def test_load_and_apply():
    table = {"nb<=256,P<=64": {"ab_group": 4, "ab_threads": 128, "ms": 0.1, "default_ms": 0.2, "contexts": 3}}
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "t.json")
        with open(p, "w") as f:
            json.dump({"classes": table}, f)
        loaded = autotune.load(p)
        assert autotune.load(os.path.join(td, "absent.json")) == {}
    c = FakeCtx(200, 200, 10)
    assert autotune.apply(c, loaded) and c.shape == (4, 128)
    other = FakeCtx(200, 1000, 10)
    assert not autotune.apply(other, loaded) and other.shape is None
    nofit = FakeCtx(200, 200, 10, fits=False)
    assert not autotune.apply(nofit, loaded)


def test_committed_table_is_well_formed():
    table = autotune.load()
    for key, e in table.items():
        assert key.startswith("nb<=") and ",P<=" in key
        assert e["ab_group"] in (1, 2, 4, 8, 16) and e["ab_threads"] in (128, 256, 512, 1024)
        assert e["ms"] > 0 and e["contexts"] >= 1
