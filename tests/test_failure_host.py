"""Failure detection made on the host, no GPU: output files and HDF5 line lists cut short raise a clean
error naming the file; a rank of a sharded synthesis that leaves between two steps is noticed by the
others before their next step (a heartbeat through the process group's store), on gloo CPU ranks."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

import helpers as H


def _truncations(path):
    size = os.path.getsize(path)
    return sorted({4, 7, size // 3, size // 2, size - 8, size - 1})


def test_truncated_output_files(tmp_path):
    from fastspec_b200 import fsio
    rng = np.random.default_rng(3)
    nwl, ntau, nmu = 50, 12, 5
    wave = np.linspace(5000, 5001, nwl)
    files = {}
    p = str(tmp_path / "fs_lineop.bin")
    fsio.write_opac(p, wave, rng.uniform(0, 1, (nwl, ntau)), *(rng.uniform(1, 2, ntau) for _ in range(5)))
    files[p] = fsio.read_opac
    p = str(tmp_path / "fs_spec.bin")
    fsio.write_spec(p, wave, np.linspace(1, 0.1, nmu), rng.uniform(0, 1, (nwl, nmu)), rng.uniform(0, 1, (nwl, nmu)))
    files[p] = fsio.read_spec
    p = str(tmp_path / "fs_flux.bin")
    fsio.write_flux(p, wave, rng.uniform(0, 1, nwl), rng.uniform(1, 2, nwl))
    files[p] = fsio.read_flux
    p = str(tmp_path / "fs_linst.bin")
    fsio.write_linst(p, np.array(["Fe"] * 20), np.ones(20, np.int32), wave[:20], rng.uniform(0, 1, 20).astype(np.float32))
    files[p] = fsio.read_linst
    for path, reader in files.items():
        whole = open(path, "rb").read()
        reader(path)                                       # the whole file reads
        for cut in _truncations(path):
            q = path + ".cut"
            with open(q, "wb") as f:
                f.write(whole[:cut])
            with pytest.raises(fsio.FsioError) as e:
                reader(q)
            assert q in str(e.value)


def test_truncated_hdf5_list(tmp_path):
    from fastspec_b200 import fsio, hdf5
    from fastspec_b200 import workloads as W
    L = W.atomic_lines(400, 5000.0, 5010.0, 5)
    t = L._txt
    path = str(tmp_path / "lines.h5")
    fsio.write_hdf5_lines(path, L.species, L.spc, L.wl, t["elo"], t["loggf"], t["lgrad"], t["lgqst"], t["lgvdw"])
    cols, attrs, units = hdf5.read_lines(path)
    assert len(cols["W"]) == 400
    whole = open(path, "rb").read()
    for cut in (16, 200, len(whole) // 2, len(whole) - 100):
        q = path + ".cut"
        with open(q, "wb") as f:
            f.write(whole[:cut])
        with pytest.raises(hdf5.HDF5Error):
            hdf5.read_lines(q)


def leaving_worker(rank, world, port, out):
    """Every rank runs sharded step 0; then rank world-1 leaves; the others check their peers before
    step 1 and record what they saw."""
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    import oracle
    from fastspec_b200 import shard
    from test_shard_gloo import OracleBackend, case
    grid, st, co, arr = case()
    backend = OracleBackend(oracle, grid, st, co, arr)
    shard.check_peers(0, timeout_s=20)
    res = shard.run(backend)
    if rank == world - 1:
        with open(out + ".left", "w") as f:
            f.write("1")
        os._exit(0)                                        # leaves between steps, no collective in flight
    try:
        shard.check_peers(1, timeout_s=3)
        seen = "none"
    except shard.PeerLost as e:
        seen = "lost:" + ",".join(str(r) for r in e.ranks)
    with open(out + ".rank%d" % rank, "w") as f:
        f.write(seen + "\n%.17g" % float(res["flux"][0].sum()))
    os._exit(0)                                            # the group cannot be torn down with a peer gone


@pytest.mark.parametrize("world", [2, 3])
def test_rank_leaving_between_steps_is_noticed(tmp_path, world):
    from test_shard_gloo import free_port
    out = str(tmp_path / "leave")
    mp.start_processes(leaving_worker, args=(world, free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    assert os.path.exists(out + ".left")
    for r in range(world - 1):
        seen, flux = open(out + ".rank%d" % r).read().split("\n")
        assert seen == "lost:%d" % (world - 1), seen
        assert np.isfinite(float(flux))
