// CTSystemElements_HF.h -- drop-in for the reference's geometry structs
// (CT_Recon/CTSystemElements_HF.h:13-151) over librecon_b200.
//
// Same struct names, field names, types and order; LoadFromConfigFile reads
// the same `key = value  # comment` files through recon_geometry_from_cfg
// (the reference parses with its vendored ConfigFile class).  A missing file
// or key throws recon_b200::config_error (the reference throws
// ConfigFile::file_not_found / key_not_found).
#pragma once

#include <stdexcept>
#include <string>

#include "recon_b200.h"

namespace recon_b200 {
struct config_error : std::runtime_error {
    recon_status_t status;
    config_error(recon_status_t s, const std::string& m) : std::runtime_error(m), status(s) {}
};

struct loaded_config {
    recon_geometry_t geom;
    recon_filepaths_t paths;
    explicit loaded_config(const std::string& path)
    {
        recon_status_t s = recon_geometry_from_cfg(path.c_str(), &geom, &paths);
        if (s != RECON_OK) throw config_error(s, recon_last_error());
    }
};
}  // namespace recon_b200

struct CalibrationParam {
    float R, Rf, Ry, Dx, Dz, xangle, yangle, zangle, M;
    int LoadFromConfigFile(std::string FilePath)
    {
        recon_b200::loaded_config c(FilePath);
        const recon_calibration_t& k = c.geom.cal;
        R = k.R; Rf = k.Rf; Ry = k.Ry; Dx = k.Dx; Dz = k.Dz;
        xangle = k.xangle; yangle = k.yangle; zangle = k.zangle; M = k.M;
        return 0;
    }
};

struct Detector {
    unsigned int NumTAxPixels;
    unsigned int NumAxPixels;
    float TAxPixDimMm;
    float AxPixDimMm;
    int LoadFromConfigFile(std::string FileName)
    {
        recon_b200::loaded_config c(FileName);
        NumTAxPixels = c.geom.det.NumTAxPixels; NumAxPixels = c.geom.det.NumAxPixels;
        TAxPixDimMm = c.geom.det.TAxPixDimMm; AxPixDimMm = c.geom.det.AxPixDimMm;
        return 0;
    }
};

struct ScanParameters {
    unsigned int N_iteration;
    unsigned int NumProj;
    float DeltaAng;
    int LoadFromConfigFile(std::string FilePath)
    {
        recon_b200::loaded_config c(FilePath);
        N_iteration = c.geom.scan.N_iteration; NumProj = c.geom.scan.NumProj; DeltaAng = c.geom.scan.DeltaAng;
        return 0;
    }
};

struct VoxVolParam {
    unsigned int Xdim, Ydim, Zdim;
    float XVoxSize, YVoxSize, ZVoxSize;
    int LoadFromConfigFile(std::string FilePath)
    {
        recon_b200::loaded_config c(FilePath);
        Xdim = c.geom.vox.Xdim; Ydim = c.geom.vox.Ydim; Zdim = c.geom.vox.Zdim;
        XVoxSize = c.geom.vox.XVoxSize; YVoxSize = c.geom.vox.YVoxSize; ZVoxSize = c.geom.vox.ZVoxSize;
        return 0;
    }
};

// ObjectParam is carried by the voxel-driven projector's signature only.
struct ObjectParam {
    float ObjX, ObjY, ObjZ, ObjXangle, ObjYangle, ObjZangle;
};

struct FilePaths {
    std::string ProjFileFolder, ProjFileNameRoot, ProjFileSuffix;
    std::string ReconFileFolder, ReconFileNameRoot, ReconFileSuffix;
    std::string sim_ObjFileFolder, sim_ObjFileName, sim_BpFileNameRoot, sim_BpFileSuffix;
    int LoadFromconfigFile(std::string FilePath)
    {
        recon_b200::loaded_config c(FilePath);
        const recon_filepaths_t& p = c.paths;
        ProjFileFolder = p.ProjFileFolder; ProjFileNameRoot = p.ProjFileNameRoot; ProjFileSuffix = p.ProjFileSuffix;
        ReconFileFolder = p.ReconFileFolder; ReconFileNameRoot = p.ReconFileNameRoot;
        ReconFileSuffix = p.ReconFileSuffix; sim_ObjFileFolder = p.ObjFileFolder; sim_ObjFileName = p.ObjFileName;
        sim_BpFileNameRoot = p.BpFileNameRoot; sim_BpFileSuffix = p.BpFileSuffix;
        return 0;
    }
};

namespace recon_b200 {
inline recon_geometry_t make_geometry(const CalibrationParam& c, const Detector& d, const VoxVolParam& v,
                                      unsigned NumProj = 0, float DeltaAng = 0.0f, unsigned N_iteration = 0)
{
    recon_geometry_t g;
    g.cal = {c.R, c.Rf, c.Ry, c.Dx, c.Dz, c.xangle, c.yangle, c.zangle, c.M};
    g.det = {d.NumTAxPixels, d.NumAxPixels, d.TAxPixDimMm, d.AxPixDimMm};
    g.vox = {v.Xdim, v.Ydim, v.Zdim, v.XVoxSize, v.YVoxSize, v.ZVoxSize};
    g.scan = {N_iteration, NumProj, DeltaAng};
    return g;
}
}  // namespace recon_b200
