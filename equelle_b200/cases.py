"""Input files for the generated-style C++ simulators (equelle_b200/sims).

Each writer puts the seeded synthetic inputs of one configuration in a
directory, as the text files the runtime's input functions read, and returns
the `key=value` arguments of the run (the generated main() turns them into
an Opm::ParameterGroup).
"""
import os

import numpy as np

from . import programs


def _write(path, values, fmt):
    np.savetxt(path, np.asarray(values).reshape(-1), fmt=fmt)
    return path


def heat(dirpath, nx=64, ny=64, steps=20, dt=0.5, seed=0, k=0.3, cv=1.0):
    """Implicit heat equation, 2D (the 64x64 configuration by default)."""
    os.makedirs(dirpath, exist_ok=True)
    grid, c = programs.heat_case(nx, ny, steps=steps, dt=dt, seed=seed)
    args = ["%s=%s" % kv for kv in grid.items()]
    args += [
        "k=%r" % k, "cv=%r" % cv,
        "u_initial_from_file=true", "u_initial_filename=" + _write(os.path.join(dirpath, "u0.txt"), c["u_initial"], "%.17g"),
        "dir_boundary_filename=" + _write(os.path.join(dirpath, "dir_faces.txt"), c["dir_faces"], "%d"),
        "dir_val_from_file=true", "dir_val_filename=" + _write(os.path.join(dirpath, "dir_val.txt"), c["dir_val"], "%.17g"),
        "timesteps_filename=" + _write(os.path.join(dirpath, "timesteps.txt"), c["timesteps"], "%.17g"),
        "abs_res_tol=1e-10", "linsolver_residual_tolerance=1e-12",
    ]
    return args


def two_phase(dirpath, nx=128, ny=128, nz=64, steps=30, dt=86400.0, seed=0, corr_len=8.0):
    """Fully implicit oil-water flow (the 128x128x64 configuration by
    default); nz=None gives the 2D variant."""
    os.makedirs(dirpath, exist_ok=True)
    grid, c = programs.two_phase_case(nx, ny, nz, steps=steps, dt=dt, seed=seed, corr_len=corr_len)
    args = ["%s=%s" % kv for kv in grid.items()]
    args += [
        "perm_from_file=true", "perm_filename=" + _write(os.path.join(dirpath, "perm.txt"), c["perm"], "%.17g"),
        "poro=0.2", "sw_initial=0.2",
        "watervisc=%r" % c["watervisc"], "oilvisc=%r" % c["oilvisc"],
        "source_cells_filename=" + _write(os.path.join(dirpath, "source_cells.txt"), c["source_cells"], "%d"),
        "source_values_from_file=true",
        "source_values_filename=" + _write(os.path.join(dirpath, "source_values.txt"), c["source_values"], "%.17g"),
        "anchor_cells_filename=" + _write(os.path.join(dirpath, "anchor_cells.txt"), c["anchor_cells"], "%d"),
        "timesteps_filename=" + _write(os.path.join(dirpath, "timesteps.txt"), c["timesteps"], "%.17g"),
    ]
    return args


def swe(dirpath, nx=4096, ny=4096, steps=200, seed=0, sigma=40.0, binary=None):
    """Explicit shallow water, 2D (the 4096x4096 configuration by default).
    Large grids are written as raw FP64 files (".f64"), which the input
    functions read without parsing text; u and v start at zero and are
    given as constants."""
    os.makedirs(dirpath, exist_ok=True)
    grid, c = programs.swe_case(nx, ny, steps=steps, seed=seed, sigma=sigma)
    if binary is None:
        binary = nx * ny > 1 << 20
    args = ["%s=%s" % kv for kv in grid.items()]
    for name in ("h_init", "b_north", "b_south", "b_east", "b_west"):
        if binary:
            path = os.path.join(dirpath, name + ".f64")
            np.asarray(c[name], dtype="<f8").tofile(path)
        else:
            path = _write(os.path.join(dirpath, name + ".txt"), c[name], "%.17g")
        args += [name + "_from_file=true", name + "_filename=" + path]
    args += ["u_init=0", "v_init=0", "cfl=%r" % c["cfl"], "num_steps=%d" % steps]
    return args


def swe_reference(dirpath, nx=64, ny=48, steps=6, dt=0.3, seed=0, sigma=5.0, d=10.0, binary=None):
    """Inputs of the reference's generated shallow-water program
    (examples/app/out_swe.cpp, from examples/dsl/swe.equelle): the same
    seeded depth and bottom as swe() on cells of size d (the program's
    default dx = dy = 10), zero initial velocity, and a list of `steps`
    time steps of `dt` (the program reads its time steps instead of
    computing a CFL step)."""
    os.makedirs(dirpath, exist_ok=True)
    grid, c = programs.swe_case(nx, ny, steps=steps, seed=seed, sigma=sigma, dx=d, dy=d)
    if binary is None:
        binary = nx * ny > 1 << 20
    args = ["%s=%s" % kv for kv in grid.items()]
    for name in ("h_init", "b_north", "b_south", "b_east", "b_west"):
        if binary:
            path = os.path.join(dirpath, name + ".f64")
            np.asarray(c[name], dtype="<f8").tofile(path)
        else:
            path = _write(os.path.join(dirpath, name + ".txt"), c[name], "%.17g")
        args += [name + "_from_file=true", name + "_filename=" + path]
    args += ["u_init=0", "v_init=0",
             "timesteps_filename=" + _write(os.path.join(dirpath, "timesteps.txt"), [dt] * steps, "%.17g")]
    return args
