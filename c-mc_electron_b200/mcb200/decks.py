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


def finfet_grid(lg_nm: float = 20.0):
    """Node coordinates (nm) of the FinFET mesh: 80 x (30 + 2 lg_nm) x 40
    cells (80 x 50 x 40 at the 20 nm gate).  x (height): 1 nm gate oxide in
    0.5 nm cells, the 30 nm fin in 0.5 nm cells, the substrate in 2 nm cells;
    y (transport): 10 nm source and drain in 2 nm cells, the channel of
    length lg_nm in 0.5 nm cells; z (width): the 10 nm fin and its 1 nm
    oxides in 0.5 nm cells, 16 nm either side in 2 nm cells."""
    h = lg_nm / 2.0
    e = h + 10.0
    x = np.concatenate([[-1.0, -0.5], np.arange(0.0, 30.0001, 0.5), np.arange(32.0, 66.0001, 2.0)])
    y = np.concatenate([np.arange(-e, -h - 1e-9, 2.0), np.arange(-h, h + 1e-4, 0.5), np.arange(h + 2.0, e + 1e-4, 2.0)])
    z = np.concatenate([np.arange(-17.0, -1.0, 2.0), [-1.0, -0.5], np.arange(0.0, 10.0001, 0.5), [10.5, 11.0],
                        np.arange(13.0, 27.0001, 2.0)])
    return x, y, z


def finfet(dirpath: str, electrons=300000, holes=50000, vd=0.7, vg=0.8, phims=-0.46, dt=2e-16, total_step=7000,
           heat_steps=3000, stat_step=1000, mr_step=50, surface_scatter=True, compute_heat=True,
           delta_nm=0.4, lambda_nm=1.5, kelvin=300.0, lg_nm=20.0, min_per_cell=(3, 1), quantum=None) -> dict:
    """The n-FinFET of the self-consistent workload, in the reference's deck
    language and with the reference FinFET's topology (finfet/ldg.txt):
    fin 30 nm tall (x) and 10 nm wide (z), gate length lg_nm (y; 20 nm by
    default), 1 nm SiO2 on the top and both sides of the gated fin, oxide
    beside the fin's foot, a silicon substrate below; source / drain 1e20
    cm^-3 donors rolling off at 2 nm per decade into a 1e15 cm^-3 p-type
    channel as 0.5 nm stair-step donor boxes; CATCH / GENERATE planes one
    cell inside the source, drain and substrate contacts, REFLECT at the fin
    ends, SCATTOX on every Si/SiO2 or outer face; contacts: source 0 V,
    drain vd, substrate 0 V, a three-plane gate at vg with work-function
    difference phims.  min_per_cell: the fewest electrons / holes of a
    silicon cell (default_par_number).  Doping values are in m^-3 as the
    reference reads them.  The surface-roughness parameters go to input.txt
    as surface_roughness_delta_nm / surface_roughness_lambda_nm (keys the
    reference does not read).  quantum = (ratio, theta_nm, eb_v, start_step):
    the effective-potential quantum correction on (Flag_QuantumCorrection,
    quantum_start_step), with an ep_parm window of ratio * theta_nm on every
    axis, oxide barrier eb_v, over the gated fin (quantumRegion)."""
    os.makedirs(dirpath, exist_ok=True)
    x, y, z = finfet_grid(lg_nm)
    write_grid(os.path.join(dirpath, "lgrid.txt"), x, y, z)
    g = lambda v: f"{v:g}"
    h = lg_nm / 2.0
    e = h + 10.0
    Y = f"{g(-e)} {g(e)}"
    L = [
        f"default_par_number {min_per_cell[0]} {min_per_cell[1]}",
        f"region -1 66 {Y} -17 27 VACUUM",
        f"region 0 30 {Y} 0 10 SILICON",
        f"region 30 66 {Y} -17 27 SILICON",
        f"region -1 0 {Y} -1 11 OXIDE",
        f"region 0 24 {Y} -1 0 OXIDE",
        f"region 0 24 {Y} 10 11 OXIDE",
        f"region 24 30 {Y} -17 0 OXIDE",
        f"region 24 30 {Y} 10 27 OXIDE",
        f"donor -1 66 {Y} -17 27 0",
        f"donor 0 24 {g(-e)} {g(-h)} 0 10 1e+26",
        f"donor 0 24 {g(h)} {g(e)} 0 10 1e+26",
    ]
    for s_ in range(int(round(h / 0.5))):  # 2 nm / decade roll-off on the 0.5 nm channel grid
        conc = 1e26 * 10.0 ** (-(0.5 * s_ + 0.25) / 2.0)
        y0, y1 = -h + 0.5 * s_, -h + 0.5 * (s_ + 1)
        L.append(f"donor 0 24 {g(y0)} {g(y1)} 0 10 {conc:.6g}")
        L.append(f"donor 0 24 {g(-y1)} {g(-y0)} 0 10 {conc:.6g}")
    c, r = e - 2.0, e - 4.0  # CATCH / GENERATE planes; contact-attached range
    L += [
        f"acceptor -1 66 {Y} -17 27 0",
        f"acceptor 0 30 {g(-h)} {g(h)} 0 10 1e+21",
        f"acceptor 24 30 {Y} 0 10 1e+21",
        f"acceptor 30 66 {Y} -17 27 1e+21",
        f"motioncube -1 66 {Y} -17 27 PASS PASS PASS PASS PASS PASS",
        f"motionplane 0 24 {g(-c)} {g(-c)} 0 10 LEFT CATCH",
        f"motionplane 0 24 {g(-c)} {g(-c)} 0 10 RIGHT GENERATE",
        f"motionplane 0 30 {g(-e)} {g(-e)} 0 10 LEFT REFLECT",
        f"motionplane 0 24 {g(c)} {g(c)} 0 10 RIGHT CATCH",
        f"motionplane 0 24 {g(c)} {g(c)} 0 10 LEFT GENERATE",
        f"motionplane 0 30 {g(e)} {g(e)} 0 10 RIGHT REFLECT",
        f"motionplane 0 0 {Y} 0 10 UP SCATTOX",
        f"motionplane 0 30 {Y} 0 0 FRONT SCATTOX",
        f"motionplane 0 30 {Y} 10 10 BACK SCATTOX",
        f"motionplane 30 30 {Y} -17 0 UP SCATTOX",
        f"motionplane 30 30 {Y} 10 27 UP SCATTOX",
        f"motionplane 30 66 {g(-e)} {g(-e)} -17 27 LEFT SCATTOX",
        f"motionplane 30 66 {g(e)} {g(e)} -17 27 RIGHT SCATTOX",
        f"motionplane 30 66 {Y} -17 -17 FRONT SCATTOX",
        f"motionplane 30 66 {Y} 27 27 BACK SCATTOX",
        f"motionplane 66 66 {Y} -17 27 DOWN SCATTOX",
        f"motionplane 64 64 {Y} -17 27 UP GENERATE",
        f"motionplane 64 64 {Y} -17 27 DOWN CATCH",
        f"attachcontact 0 30 {Y} 0 10 0",
        f"attachcontact 0 24 {g(-e)} {g(-r)} 0 10 1",
        f"attachcontact 0 24 {g(r)} {g(e)} 0 10 2",
        f"attachcontact 60 66 {Y} -17 27 3",
        "surfaces 3",
        "0 0 0",
        "2 0 4",
        "2 10 5",
        f"surface_scatter_range 0 24 {Y} 0 10",
        "contact", "1 0", f"0 24 {g(-e)} {g(-e)} 0 10", "0",
        "contact", "1 0", f"0 24 {g(e)} {g(e)} 0 10", g(vd),
        "contact", "1 0", f"66 66 {Y} -17 27", "0",
        "contact", f"3 {g(phims)}", f"-1 -1 {g(-h)} {g(h)} -1 11", f"-1 24 {g(-h)} {g(h)} -1 -1",
        f"-1 24 {g(-h)} {g(h)} 11 11", g(vg),
    ]
    if quantum is not None:
        r, t, eb = (g(v) for v in quantum[:3])
        L += [f"ep_parm {r} {t} {r} {t} {r} {t} {eb}", f"quantumRegion 0 24 {Y} 0 10"]
    L.append("end")
    with open(os.path.join(dirpath, "ldg.txt"), "w") as f:
        f.write("\n".join(L) + "\n")
    write_input(os.path.join(dirpath, "input.txt"), dt=dt, Temperature=kelvin, total_step=total_step,
                ElectronNumber=electrons, HoleNumber=holes, Flag_SurfaceScatter=int(surface_scatter),
                Flag_MultipleRefresh=1, mr_step=mr_step, Flag_compute_heat=int(compute_heat), heat_steps=heat_steps,
                stat_step=stat_step, stat_heat_step=stat_step, surface_roughness_delta_nm=delta_nm,
                surface_roughness_lambda_nm=lambda_nm,
                **({} if quantum is None else dict(Flag_QuantumCorrection=1, quantum_start_step=int(quantum[3]))))
    return dict(input=os.path.join(dirpath, "input.txt"), grid=os.path.join(dirpath, "lgrid.txt"),
                device=os.path.join(dirpath, "ldg.txt"))
