"""IDL ascii ``.out`` plot files (src/ModWritePlotIdl.f90 format).

Header (one item per line):
  1. unit/heading string ("normalized variables")
  2. nStep, time, nDim (negative for non-uniform grids), nParam, nVar
  3. grid size per dimension
  4. the nParam parameter values (gamma, ...)
  5. names of coordinates, variables and parameters
Then one row per cell: coordinates followed by the nVar values.
"""
import numpy as np


def read_idl_ascii(path):
    with open(path) as f:
        head = f.readline().strip()
        p = f.readline().split()
        nstep, time, ndim, npar, nvar = int(p[0]), float(p[1]), int(p[2]), int(p[3]), int(p[4])
        size = [int(x) for x in f.readline().split()]
        params = [float(x) for x in f.readline().split()] if npar > 0 else []
        names = f.readline().split()
        data = np.loadtxt(f)
    ncoord = abs(ndim)
    return {
        "heading": head, "nStep": nstep, "time": time, "nDim": ndim,
        "size": size, "params": params, "names": names,
        "coord": data[:, :ncoord], "var": data[:, ncoord:ncoord + nvar],
        "varnames": names[ncoord:ncoord + nvar],
    }


def write_idl_ascii(path, coord, var, coord_names, var_names, nstep, time,
                    params=(), param_names=(), heading="normalized variables"):
    coord = np.atleast_2d(np.asarray(coord))
    if coord.shape[0] != len(var):
        coord = coord.T
    ndim = coord.shape[1]
    with open(path, "w") as f:
        f.write(heading + "\n")
        f.write("%10d %17.10E %2d %2d %2d\n" % (nstep, time, -ndim, len(params), len(var_names)))
        f.write("%8d\n" % len(var))
        if params:
            f.write(" ".join("%17.10E" % p for p in params) + "\n")
        f.write(" ".join(list(coord_names) + list(var_names) + list(param_names)) + "\n")
        for c, v in zip(coord, var):
            f.write(" ".join("%17.10E" % x for x in list(c) + list(v)) + "\n")
