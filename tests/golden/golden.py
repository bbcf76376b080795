"""Golden fixtures: small cases run through the reference's own kernel sources.

Each fixture (``<name>.npz``) stores the complete inputs of a case and the fields the
reference's kernels (oracle/_ref, launch for launch as Engine.py) produce after
``nsteps`` steps.  They are made by ``make_golden.py`` in this directory.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_FIELDS = ("z", "u", "v", "t_z", "t_u", "t_v", "H_moi", "khouot", "FS", "tFS", "dH", "Htdu", "Htdv",
              "VTH", "Kx", "Ky", "Qbx", "Qby", "ubt", "ubp", "vbt", "vbd", "hi",
              "daui", "cuoii", "moci", "dauj", "cuoij", "mocj")


def save(path, case, outputs):
    from hydist.params import HydCaseParams
    p = case.params
    d = {"N": case.N, "M": case.M, "total_time": case.total_time, "nsteps": case.nsteps,
         "t_start": case.t_start, "boundary_type": case.boundary_type,
         "params": np.frombuffer(bytes(p), dtype=np.uint8).copy()}
    for k, v in case.fields.items():
        d["in_" + k] = v
    for e in range(4):
        d["table_%d" % e] = case.tables[e]
        d["cc_%d" % e] = case.cc[e]
    for k, v in outputs.items():
        d["out_" + k] = v
    np.savez_compressed(path, **d)


def load(name):
    from hydist.cases import Case
    from hydist.params import HydCaseParams
    z = np.load(os.path.join(HERE, name + ".npz"))
    from hydist.params import default_params
    # fixtures store the struct as it was when they were made: the reference's constants
    # and run options; fields added since (the morphodynamic options) keep their defaults
    p = default_params()
    raw = z["params"].tobytes()
    ctypes.memmove(ctypes.addressof(p), raw, min(len(raw), ctypes.sizeof(p)))
    fields = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    case = Case(name, int(z["N"]), int(z["M"]), p, fields, z["boundary_type"],
                [z["table_%d" % e] for e in range(4)], [z["cc_%d" % e] for e in range(4)],
                int(z["total_time"]), float(z["t_start"]), int(z["nsteps"]))
    outputs = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return case, outputs


def names():
    return sorted(f[:-4] for f in os.listdir(HERE) if f.endswith(".npz"))
