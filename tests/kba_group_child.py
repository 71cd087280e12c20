"""One process of the node-group test (started by minisweep_b200.launch):
for several process grids, the library's Quantities_create (an allgather of
the subdomain sizes) and get_state_norms (a sum over the active processes)
through the node group's shared-memory collectives, no GPU needed.  Writes
its results to <out_dir>/proc_<i>.json."""
import ctypes
import json
import os
import sys

import numpy as np

import minisweep_b200 as msb

GRIDS = [(1, 1), (2, 2), (2, 1), (1, 3), (4, 1), (2, 2)]
GX, GY, NZ, NE, NM, NA = 9, 6, 2, 3, 4, 8


def main(out_dir):
    L = msb.lib()
    env = msb.Env()
    L.Env_initialize(ctypes.byref(env), 0, None)
    proc = int(os.environ["MSB_PROC"])
    res = {"proc": env.proc_, "nproc": env.nproc_world_, "runs": []}
    DP = ctypes.POINTER(ctypes.c_double)
    for npx, npy in GRIDS:
        args = msb.Arguments()
        L.Arguments_create_from_string(ctypes.byref(args), f"--nproc_x {npx} --nproc_y {npy}".encode())
        L.Env_set_values(ctypes.byref(env), ctypes.byref(args))
        L.Arguments_destroy(ctypes.byref(args))
        if not L.Env_is_proc_active(ctypes.byref(env)):
            res["runs"].append(None)
            continue
        _, nx = msb.local_extent(GX, npx, proc % npx)
        _, ny = msb.local_extent(GY, npy, proc // npx)
        dims = msb.Dimensions(nx, ny, NZ, NE, NM, NA)
        q = msb.Quantities()
        L.Quantities_create(ctypes.byref(q), dims, ctypes.byref(env))
        v = np.zeros(nx * ny * NZ * NE * NM * 4)
        L.initialize_state(v.ctypes.data_as(DP), dims, 4, ctypes.byref(q))
        s, d = ctypes.c_double(), ctypes.c_double()
        L.get_state_norms(v.ctypes.data_as(DP), np.zeros_like(v).ctypes.data_as(DP), dims, 4, ctypes.byref(s),
                          ctypes.byref(d), ctypes.byref(env))
        res["runs"].append([q.ix_base, q.iy_base, q.ncell_x_g, q.ncell_y_g, d.value])
        L.Quantities_destroy(ctypes.byref(q))
    L.Env_finalize(ctypes.byref(env))
    with open(os.path.join(out_dir, f"proc_{proc}.json"), "w") as f:
        json.dump(res, f)


if __name__ == "__main__":
    main(sys.argv[1])
