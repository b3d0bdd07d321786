"""Multi-GPU sharding on the CPU: two gloo ranks, each filling its slice of every stream.

bench.py's multi-GPU mode gives rank r the outputs [r*n, (r+1)*n) of one stream by setting
the generator's offset to the engine position of output r*n (bench.rank_stream); there is
no data collective.  Here two ranks do exactly that with the oracle (the reference's
semantics), gather their slices, and rank 0 checks that the concatenation equals one
generator producing 2n outputs -- counter engines (Philox, ThreeFry) with one- and two-word
distributions, stateful engines (XORWOW, MRG32k3a, LFSR113) with one-word ones.  Where no
offset selects the slice (MT19937, MTGP32; a stateful engine consuming two values per output, whose
offsets rotate engines by values, not outputs -- checked here too) the ranks use distinct
seeds, and the test checks their streams differ.
"""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench
from oracle import pyorc

CASES = [(404, "uniform"), (404, "uniform_double"), (410, "uint"), (410, "normal"),
         (401, "uniform"), (402, "uniform"), (406, "uint")]
SEEDED = [(407, "uint"), (403, "uniform"), (401, "uniform_double"), (402, "normal")]
N = 3 * 131072 + 1000  # crosses the stateful engines' slot boundary


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, failures):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        orc = pyorc.CLib("orc")
        for rng, d in CASES:
            seed, off = bench.rank_stream(rng, d, rank, N)
            assert seed == bench.SEED and off is not None
            params = (0.0, 1.0) if "normal" in d else ()
            st, mine = pyorc.run_sequence(orc, rng, seed, off, [(d, N, params, 0)])[0]
            assert st == 0
            t = torch.from_numpy(mine.view(np.uint8).copy())
            parts = [torch.empty_like(t) for _ in range(world)]
            dist.all_gather(parts, t)
            if rank == 0:
                whole = pyorc.run_sequence(orc, rng, bench.SEED, 0, [(d, world * N, params, 0)])[0][1]
                got = torch.cat(parts).numpy()
                if not np.array_equal(got, whole.view(np.uint8)):
                    failures.append((rng, d))
        for rng, d in SEEDED:
            seed, off = bench.rank_stream(rng, d, rank, N)
            assert off is None and seed == bench.SEED + rank
            params = (0.0, 1.0) if "normal" in d else ()
            st, mine = pyorc.run_sequence(orc, rng, seed, None, [(d, 4096, params, 0)])[0]
            t = torch.from_numpy(mine.view(np.uint8).copy())
            parts = [torch.empty_like(t) for _ in range(world)]
            dist.all_gather(parts, t)
            if rank == 0 and torch.equal(parts[0], parts[1]):
                failures.append((rng, d))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_slices_concatenate_to_one_stream():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        failures = m.list()
        mp.start_processes(_rank, args=(2, _free_port(), failures), nprocs=2, join=True,
                           start_method="spawn")
        assert list(failures) == []
