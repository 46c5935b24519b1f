"""Shared helpers for tests: writing reference-format configuration files and
per-view projection files."""
import os

import numpy as np

from oracle import oracle as O
from recon_b200.configs import geom_dict
from recon_b200.phantom import noisy, phantom


def write_cfg(path, cfg, proj_folder, recon_folder, obj_folder="", obj_name="object.bin"):
    """A configuration file in the reference's key = value format
    (CT_Recon/MasterParameterFile.origin)."""
    lines = [
        "# test configuration",
        f"R = {cfg['R']}   # mm", f"Rf = {cfg['Rf']}", f"Ry = {cfg['Ry']}", f"Dx = {cfg['Dx']}",
        f"Dz = {cfg['Dz']}", f"xangle = {cfg['xangle']}", f"yangle = {cfg['yangle']}",
        f"zangle = {cfg['zangle']}", f"M = {cfg['M']}", "",
        f"TAxPixels = {cfg['TAxPixels']}", f"AxPixels = {cfg['AxPixels']}",
        f"TAxPixDim = {cfg['TAxPixDim']}", f"AxPixDim = {cfg['AxPixDim']}", "",
        f"Xdim = {cfg['Xdim']}", f"Ydim = {cfg['Ydim']}", f"Zdim = {cfg['Zdim']}",
        f"XVoxSize = {cfg['XVoxSize']}", f"YVoxSize = {cfg['YVoxSize']}", f"ZVoxSize = {cfg['ZVoxSize']}", "",
        f"N_iteration = {cfg['N_iteration']}", f"NumProj = {cfg['NumProj']}",
        f"DeltaAng = {float(np.float32(cfg['DeltaAng'])):.9g}", "",
        f"ProjFileFolder = {proj_folder}", "ProjFileNameRoot = proj", "ProjFileSuffix = .bin",
        f"ReconFileFolder = {recon_folder}", "ReconFileNameRoot = recon", "ReconFileSuffix = .bin", "",
        f"ObjFileFolder = {obj_folder}", f"ObjFileName = {obj_name}", "BpFileNameRoot = bp",
        "BpFileSuffix = .bin",
    ]
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def write_case(tmp_path, cfg, seed=0, I0=1e5):
    """Phantom -> FP64 line integrals -> Poisson noise -> per-view files
    proj_<n>.bin in a new folder; returns the folder."""
    folder = os.path.join(str(tmp_path), "case")
    os.makedirs(folder, exist_ok=True)
    g = O.Geom.from_dict(geom_dict(cfg))
    vol = phantom(cfg, seed=seed, n_ellipsoids=6)
    nproj = int(cfg["NumProj"])
    p = O.x_fp_all(g, nproj, np.float32(cfg["DeltaAng"]), vol.astype(np.float64).ravel())
    gs = noisy(p, I0, seed).reshape(nproj, -1)
    for n in range(nproj):
        gs[n].astype(np.float32).tofile(os.path.join(folder, f"proj_{n}.bin"))
    vol.astype(np.float32).tofile(os.path.join(folder, "object.bin"))
    return folder
