"""Writers for the reference's input decks (input.txt, lgrid.txt, ldg.txt).

The formats are the reference's: input.txt is `key=value` lines read by
MeshQuantities::getInputData (src/mcmodel.cpp:3824-3992); lgrid.txt lists the
node coordinates per axis in micrometres (read_grid_file, :4595-4693);
ldg.txt is the device script of read_device_file (:4190-4584), coordinates in
nanometres aligned to grid nodes, doping in m^-3.  These writers produce the
synthetic workloads the engine is measured on.
"""
from __future__ import annotations

import os

import numpy as np


def write_grid(path: str, x_nm, y_nm, z_nm):
    with open(path, "w") as f:
        for axis in (x_nm, y_nm, z_nm):
            f.write(f"{len(axis)}\n")
            for v in axis:
                f.write(f"{v * 1e-3:.10g}\n")


def write_input(path: str, **kv):
    defaults = dict(gridFile="lgrid.txt", device_file_name="ldg.txt", total_step=100, ElectronNumber=100000,
                    HoleNumber=100000, Temperature=300, dt=1e-15, stat_step=1000000, stat_heat_step=1000000,
                    NonLinearPoisson=0, Flag_QuantumCorrection=0, Flag_MultipleRefresh=0, Flag_compute_potential=1,
                    Flag_compute_heat=0, Flag_SurfaceScatter=0, heat_steps=0, mr_step=50, valley=1,
                    Flag_restart=0, OutPut_DIR="./data")
    defaults.update(kv)
    with open(path, "w") as f:
        for k, v in defaults.items():
            f.write(f"{k}={v}\n")


def contact_bar(dirpath: str, nx=8, ny=10, nz=6, cell_nm=5.0, donor_m3=1e24, vd=0.3, electrons=4000, holes=0,
                dt=1e-15, kelvin=300.0, surfaces=False) -> dict:
    """n-Si bar with a grounded contact on the y = 0 node plane and a contact
    at `vd` volts on the far y plane (REFLECT on every face): the smallest
    device with Dirichlet rows in its Poisson problem.  surfaces=True adds
    Si/SiO2 surfaces at x = 0 and z = 0 with surface scattering in the whole
    bar (the `surfaces` and `surface_scatter_range` keywords)."""
    os.makedirs(dirpath, exist_ok=True)
    X, Y, Z = nx * cell_nm, ny * cell_nm, nz * cell_nm
    write_grid(os.path.join(dirpath, "lgrid.txt"), np.arange(nx + 1) * cell_nm, np.arange(ny + 1) * cell_nm,
               np.arange(nz + 1) * cell_nm)
    g = lambda v: f"{v:g}"
    box = f"0 {g(X)} 0 {g(Y)} 0 {g(Z)}"
    lines = [
        "default_par_number 1 0",
        f"region {box} SILICON",
        f"donor {box} {donor_m3:g}",
        f"acceptor {box} 0",
        f"motioncube {box} PASS PASS PASS PASS PASS PASS",
        f"motionplane 0 0 0 {g(Y)} 0 {g(Z)} UP REFLECT",
        f"motionplane {g(X)} {g(X)} 0 {g(Y)} 0 {g(Z)} DOWN REFLECT",
        f"motionplane 0 {g(X)} 0 0 0 {g(Z)} LEFT REFLECT",
        f"motionplane 0 {g(X)} {g(Y)} {g(Y)} 0 {g(Z)} RIGHT REFLECT",
        f"motionplane 0 {g(X)} 0 {g(Y)} 0 0 FRONT REFLECT",
        f"motionplane 0 {g(X)} 0 {g(Y)} {g(Z)} {g(Z)} BACK REFLECT",
        "contact", "1 0", f"0 {g(X)} 0 0 0 {g(Z)}", "0",
        "contact", "1 0", f"0 {g(X)} {g(Y)} {g(Y)} 0 {g(Z)}", f"{vd:g}",
    ]
    if surfaces:
        lines += ["surfaces 2", "0 0 0", "2 0 4", f"surface_scatter_range {box}"]
    lines.append("end")
    with open(os.path.join(dirpath, "ldg.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    write_input(os.path.join(dirpath, "input.txt"), dt=dt, Temperature=kelvin, Flag_SurfaceScatter=int(surfaces),
                ElectronNumber=electrons, HoleNumber=holes)
    return dict(input=os.path.join(dirpath, "input.txt"), grid=os.path.join(dirpath, "lgrid.txt"),
                device=os.path.join(dirpath, "ldg.txt"))


def bulk_box(dirpath: str, nx=40, ny=20, nz=20, cell_nm=5.0, donor_m3=1e23, electrons=20000, holes=0,
             min_electrons=1, min_holes=0, dt=1e-15, kelvin=300.0) -> dict:
    """n-Si box of nx*ny*nz cubic cells, uniform donors, REFLECT on all six faces
    (the bulk frozen-field workload).  The reference's initialiser puts
    int(share * electrons) + 1 electrons and int(share * holes) + 1 holes in
    every silicon cell (compute_par_num, src/particle_init.cpp:17-74).
    Returns the deck paths."""
    os.makedirs(dirpath, exist_ok=True)
    X, Y, Z = nx * cell_nm, ny * cell_nm, nz * cell_nm
    write_grid(os.path.join(dirpath, "lgrid.txt"), np.arange(nx + 1) * cell_nm, np.arange(ny + 1) * cell_nm,
               np.arange(nz + 1) * cell_nm)
    g = lambda v: f"{v:g}"
    box = f"0 {g(X)} 0 {g(Y)} 0 {g(Z)}"
    lines = [
        f"default_par_number {min_electrons} {min_holes}",
        f"region {box} SILICON",
        f"donor {box} {donor_m3:g}",
        f"acceptor {box} 0",
        f"motioncube {box} PASS PASS PASS PASS PASS PASS",
        f"motionplane 0 0 0 {g(Y)} 0 {g(Z)} UP REFLECT",
        f"motionplane {g(X)} {g(X)} 0 {g(Y)} 0 {g(Z)} DOWN REFLECT",
        f"motionplane 0 {g(X)} 0 0 0 {g(Z)} LEFT REFLECT",
        f"motionplane 0 {g(X)} {g(Y)} {g(Y)} 0 {g(Z)} RIGHT REFLECT",
        f"motionplane 0 {g(X)} 0 {g(Y)} 0 0 FRONT REFLECT",
        f"motionplane 0 {g(X)} 0 {g(Y)} {g(Z)} {g(Z)} BACK REFLECT",
        "end",
    ]
    with open(os.path.join(dirpath, "ldg.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    write_input(os.path.join(dirpath, "input.txt"), dt=dt, Temperature=kelvin, Flag_SurfaceScatter=0,
                ElectronNumber=electrons, HoleNumber=holes)
    return dict(input=os.path.join(dirpath, "input.txt"), grid=os.path.join(dirpath, "lgrid.txt"),
                device=os.path.join(dirpath, "ldg.txt"))
