"""Device-side inputs of one solve, packed as `jaxdd_b200.batch.run` packs them, for tests that
call the C ABI directly."""

import numpy as np

from jaxdd_b200 import _lib
from jaxdd_b200.batch import _gpu, descriptor, initial_state


def pack(batch, lists):
    """Every device `k` at the ascending voltages `lists[k]`, started at its pre-bias (or first
    voltage): `(g, desc, volts, keep, offsets, counts, nflat)`; `keep` holds the tensors the
    descriptors point at."""
    import torch
    Bp, npmax = batch["Bp"], batch["np_max"]
    y0 = np.zeros((npmax + 2, 3, Bp))
    counts = np.zeros(Bp, dtype=np.int32)
    for k, dev in enumerate(batch["devices"]):
        lane = batch["lane_of"][k]
        first = dev.V_pre if dev.pre_cond else lists[k][0]
        y0[:len(dev.x), :, lane] = initial_state(dev, float(first))
        counts[lane] = len(lists[k])
    offsets = np.zeros(Bp, dtype=np.int32)
    offsets[1:] = np.cumsum(counts)[:-1]
    flat = np.zeros(max(int(counts.sum()), 1))
    for k in range(batch["n"]):
        lane = batch["lane_of"][k]
        flat[offsets[lane]:offsets[lane] + counts[lane]] = lists[k]
    g = _gpu(batch)
    cuda = torch.device("cuda")
    keep = {"y0": torch.from_numpy(y0).to(cuda), "v": torch.from_numpy(flat).to(cuda),
            "off": torch.from_numpy(offsets).to(cuda), "cnt": torch.from_numpy(counts).to(cuda)}
    desc = descriptor(batch, g, keep["y0"])
    volts = _lib.DdVoltages(keep["v"].data_ptr(), keep["off"].data_ptr(),
                            keep["cnt"].data_ptr())
    return g, desc, volts, keep, offsets, counts, flat.size
