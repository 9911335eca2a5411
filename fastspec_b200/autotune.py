"""Tile-shape choice for the batched synthesis, cached by workload signature.

The candidates (wing-pass tile width 64 or 128 wavelengths, 1 or 2 persistent CTAs per SM for the
wing pass, 2/4/8 per SM for the core pass) are timed on the batch itself by fsg_batch_tune; the
winner is kept in a JSON file keyed by the device and the batch's shape, so that later runs of a
batch of the same shape skip the timing and capture their graph with the cached choice."""
import json
import os


def signature(batch, device_name=""):
    """Key of a batch: device, number of atmospheres, their depth and wavelength counts (sums and
    maxima) and the number of candidate lines (rounded to 2 significant figures)."""
    ctx = batch.contexts
    nt = [c.ntau for c in ctx]
    nw = [c.nwl for c in ctx]
    nl = batch.lines.n
    r = lambda x: float("%.2g" % x)
    return "%s|natm=%d|ntau=%d/%d|nwl=%s/%d|lines=%s" % (device_name, len(ctx), max(nt), sum(nt), r(sum(nw)),
                                                         max(nw), r(nl))


def load(path):
    if path and os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def tuned(batch, path=None, device_name=""):
    """Apply the cached tuning of this batch's signature, or time the candidates and cache the
    winner.  Returns (tuning dict, 'cache' | 'timed')."""
    key = signature(batch, device_name)
    cache = load(path)
    if key in cache:
        batch.set_tuning(cache[key])
        return cache[key], "cache"
    t = batch.tune()
    if path:
        cache[key] = t
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    return t, "timed"
