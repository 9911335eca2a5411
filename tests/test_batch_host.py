"""Host side of the batched synthesis: the batched grid of atmospheres and the tuning cache."""
import numpy as np

from fastspec_b200 import autotune
from fastspec_b200 import workloads as W


def test_batch_grid_distributions():
    g = W.batch_grid(64)
    nt = np.array([a["ntau"] for a in g])
    assert nt.min() >= 48 and nt.max() <= 80
    span = np.array([a["grid"]["wend"] - a["grid"]["wstart"] for a in g])
    assert span.min() >= 20 and span.max() <= 200
    assert all(3000 <= a["grid"]["wstart"] and a["grid"]["wend"] <= 9000 for a in g)
    teff = np.array([a["teff"] for a in g])
    assert teff.min() >= 3800 and teff.max() <= 7500
    for a in g[:4]:
        st = a["state"]
        assert st["fractionpf"].shape == (a["ntau"], 6) and np.all(np.isfinite(st["fractionpf"]))
        assert np.all(np.diff(st["rhox"]) > 0) and np.all(st["T"] > 0)
        assert a["cont"]["cont_opac"].shape == (len(a["cont"]["cont_wave"]), a["ntau"])
    # deterministic
    h = W.batch_grid(2)
    assert np.array_equal(h[1]["state"]["fractionpf"], g[1]["state"]["fractionpf"])


class FakeBatch:
    class C:
        def __init__(self, ntau, nwl):
            self.ntau, self.nwl = ntau, nwl

    class L:
        n = 2_000_000

    def __init__(self):
        self.contexts = [self.C(60, 1000), self.C(80, 3000)]
        self.lines = self.L()
        self.timed = 0
        self.applied = None

    def tune(self):
        self.timed += 1
        return {"tile_pix": 128, "wing_ctas": 148, "core_ctas": 592, "ms_wing": 1.0, "ms_core": 0.5}

    def set_tuning(self, t):
        self.applied = t


def test_tuning_cache(tmp_path):
    path = str(tmp_path / "tune.json")
    b = FakeBatch()
    t, how = autotune.tuned(b, path, "B200")
    assert how == "timed" and b.timed == 1
    b2 = FakeBatch()
    t2, how2 = autotune.tuned(b2, path, "B200")
    assert how2 == "cache" and b2.timed == 0 and b2.applied == t
    b3 = FakeBatch()
    b3.contexts[0].ntau = 70                 # another shape: timed again
    _, how3 = autotune.tuned(b3, path, "B200")
    assert how3 == "timed"
