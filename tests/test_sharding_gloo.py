"""Multi-GPU sharding on the CPU: two gloo ranks, each filling its slice of every stream.

bench.py's multi-GPU mode gives rank r the outputs [r*n, (r+1)*n) of one stream by
positioning its generator at output r*n (bench.rank_stream, rocrand_b200_set_output_position);
there is no data collective.  The position is, by definition, the state one generator
reaches by writing r*n outputs of that kind from offset 0.  Here two ranks reach it on the
oracle (the reference's semantics) that way -- by a first call of r*n outputs -- gather the
slices they write next, and rank 0 checks that the concatenation equals one generator
producing 2n outputs: counter engines (Philox, ThreeFry) and stateful engines (XORWOW,
MRG32k3a, LFSR113) with one- and two-value distributions.  (tests/test_output_position_gpu.py
checks that the library's position equals that state.)  MT19937 and MTGP32 have no position:
the ranks use distinct seeds, and the test checks their streams differ.
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
         (401, "uniform"), (402, "uniform"), (406, "uint"), (401, "uniform_double"), (402, "normal"),
         (406, "normal_double")]
SEEDED = [(407, "uint"), (403, "uniform")]
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
            seed, pos = bench.rank_stream(rng, d, rank, N)
            assert seed == bench.SEED and pos == rank * N
            params = (0.0, 1.0) if "normal" in d else ()
            # the state after `pos` outputs of this kind, then this rank's slice
            calls = ([(d, pos, params, 0)] if pos else []) + [(d, N, params, 0)]
            res = pyorc.run_sequence(orc, rng, seed, 0, calls)
            assert all(st == 0 for st, _ in res)
            mine = res[-1][1]
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
