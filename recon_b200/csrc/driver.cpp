// driver.cpp -- host side of the reference's file-driven entry points:
// configuration parsing, raw float32 file IO and the siddon_recon drivers
// (a0_RECON_MLEM, a1_FORWARD_PROJECTION, a1_BACKWARD_PROJECTION), built on
// the C ABI.  Nothing here exits or prompts: every failure is a status code
// with a message (the reference prints and returns, throws from the parser, or
// asks on stdin whether to create a missing directory).
#include <cuda_runtime.h>
#include <sys/stat.h>
#include <sys/types.h>

#include <cerrno>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/recon_b200.h"

namespace rb {
void set_error(const std::string& msg);
recon_status_t fail(recon_status_t code, const std::string& msg);
}  // namespace rb

namespace {

using rb::fail;

// ---- configuration file ------------------------------------------------------------
//
// Format of CT_Recon/ConfigFile.cpp:67-141 (parser v2.1 by R. Wagner, vendored
// by the reference): "key = value", text after '#' is a comment, keys and
// values are trimmed, a later key replaces an earlier one, a value may
// continue on following lines that hold no '=' (up to a blank line), and a
// line containing "EndConfigFile" ends the file.

const char* kWhitespace = " \n\t\v\r\f";

std::string trimmed(const std::string& s)
{
    size_t a = s.find_first_not_of(kWhitespace);
    if (a == std::string::npos) return std::string();
    size_t b = s.find_last_not_of(kWhitespace);
    return s.substr(a, b - a + 1);
}

std::string strip_comment(const std::string& s)
{
    size_t p = s.find('#');
    return p == std::string::npos ? s : s.substr(0, p);
}

recon_status_t parse_config(const std::string& path, std::map<std::string, std::string>& kv)
{
    std::ifstream in(path.c_str());
    if (!in) return fail(RECON_ERR_FILE_NOT_FOUND, "configuration file not found: " + path);
    const std::string sentry = "EndConfigFile";
    std::string pending;  // a line read ahead while collecting a value
    bool have_pending = false;
    while (have_pending || in) {
        std::string line;
        if (have_pending) {
            line = pending;
            have_pending = false;
        } else if (!std::getline(in, line)) {
            break;
        }
        line = strip_comment(line);
        if (line.find(sentry) != std::string::npos) return RECON_OK;
        size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        std::string key = trimmed(line.substr(0, eq));
        std::string value = line.substr(eq + 1);
        // continuation lines
        std::string next;
        while (in && std::getline(in, next)) {
            if (trimmed(next).empty()) {  // blank line ends the value
                break;
            }
            std::string body = strip_comment(next);
            if (body.find('=') != std::string::npos || body.find(sentry) != std::string::npos) {
                pending = next;
                have_pending = true;
                break;
            }
            if (!trimmed(body).empty()) value += "\n";
            value += body;
        }
        kv[key] = trimmed(value);
    }
    return RECON_OK;
}

recon_status_t get_string(const std::map<std::string, std::string>& kv, const char* key, std::string& out)
{
    auto it = kv.find(key);
    if (it == kv.end()) return fail(RECON_ERR_KEY_NOT_FOUND, std::string("configuration key not found: ") + key);
    out = it->second;
    return RECON_OK;
}

template <class T>
recon_status_t get_number(const std::map<std::string, std::string>& kv, const char* key, T& out)
{
    std::string s;
    recon_status_t st = get_string(kv, key, s);
    if (st != RECON_OK) return st;
    std::istringstream is(s);
    T v{};
    if (!(is >> v)) return fail(RECON_ERR_INVALID_ARGUMENT, std::string("value of ") + key + " is not a number: " + s);
    out = v;
    return RECON_OK;
}

#define RB_TRY(x)                          \
    do {                                   \
        recon_status_t s_ = (x);           \
        if (s_ != RECON_OK) return s_;     \
    } while (0)

recon_status_t load_geometry(const std::map<std::string, std::string>& kv, recon_geometry_t& g)
{
    // CalibrationParam::LoadFromConfigFile (CTSystemElements_HF.h:25-39)
    RB_TRY(get_number(kv, "R", g.cal.R));
    RB_TRY(get_number(kv, "Rf", g.cal.Rf));
    RB_TRY(get_number(kv, "Ry", g.cal.Ry));
    RB_TRY(get_number(kv, "Dx", g.cal.Dx));
    RB_TRY(get_number(kv, "Dz", g.cal.Dz));
    RB_TRY(get_number(kv, "xangle", g.cal.xangle));
    RB_TRY(get_number(kv, "yangle", g.cal.yangle));
    RB_TRY(get_number(kv, "zangle", g.cal.zangle));
    RB_TRY(get_number(kv, "M", g.cal.M));
    // Detector (:49-57)
    RB_TRY(get_number(kv, "TAxPixels", g.det.NumTAxPixels));
    RB_TRY(get_number(kv, "AxPixels", g.det.NumAxPixels));
    RB_TRY(get_number(kv, "TAxPixDim", g.det.TAxPixDimMm));
    RB_TRY(get_number(kv, "AxPixDim", g.det.AxPixDimMm));
    // VoxVolParam (:87-98)
    RB_TRY(get_number(kv, "Xdim", g.vox.Xdim));
    RB_TRY(get_number(kv, "Ydim", g.vox.Ydim));
    RB_TRY(get_number(kv, "Zdim", g.vox.Zdim));
    RB_TRY(get_number(kv, "XVoxSize", g.vox.XVoxSize));
    RB_TRY(get_number(kv, "YVoxSize", g.vox.YVoxSize));
    RB_TRY(get_number(kv, "ZVoxSize", g.vox.ZVoxSize));
    // ScanParameters (:67-75)
    RB_TRY(get_number(kv, "N_iteration", g.scan.N_iteration));
    RB_TRY(get_number(kv, "NumProj", g.scan.NumProj));
    RB_TRY(get_number(kv, "DeltaAng", g.scan.DeltaAng));
    return RECON_OK;
}

recon_status_t copy_path(const std::string& s, char (&dst)[RECON_PATH_MAX], const char* key)
{
    if (s.size() >= RECON_PATH_MAX) return fail(RECON_ERR_INVALID_ARGUMENT, std::string(key) + " is too long");
    std::memcpy(dst, s.c_str(), s.size() + 1);
    return RECON_OK;
}

struct Paths {
    std::string ProjFileFolder, ProjFileNameRoot, ProjFileSuffix, ReconFileFolder, ReconFileNameRoot,
        ReconFileSuffix, ObjFileFolder, ObjFileName, BpFileNameRoot, BpFileSuffix;
};

recon_status_t load_paths(const std::map<std::string, std::string>& kv, Paths& p)
{
    // FilePaths::LoadFromconfigFile (CTSystemElements_HF.h:136-150)
    RB_TRY(get_string(kv, "ProjFileFolder", p.ProjFileFolder));
    RB_TRY(get_string(kv, "ProjFileNameRoot", p.ProjFileNameRoot));
    RB_TRY(get_string(kv, "ProjFileSuffix", p.ProjFileSuffix));
    RB_TRY(get_string(kv, "ReconFileFolder", p.ReconFileFolder));
    RB_TRY(get_string(kv, "ReconFileNameRoot", p.ReconFileNameRoot));
    RB_TRY(get_string(kv, "ReconFileSuffix", p.ReconFileSuffix));
    RB_TRY(get_string(kv, "ObjFileFolder", p.ObjFileFolder));
    RB_TRY(get_string(kv, "ObjFileName", p.ObjFileName));
    RB_TRY(get_string(kv, "BpFileNameRoot", p.BpFileNameRoot));
    RB_TRY(get_string(kv, "BpFileSuffix", p.BpFileSuffix));
    return RECON_OK;
}

// correct_folder_path (hf_cpp_functions.hpp:160-175): backslashes become
// slashes and a non-empty folder gets a trailing slash.
void correct_folder(std::string& f)
{
    if (f.empty()) return;
    for (char& c : f)
        if (c == '\\') c = '/';
    if (f.back() != '/') f.push_back('/');
}

// m_correct_filepaths (hf_siddon_recon.hpp:347-357)
void correct_paths(Paths& p)
{
    correct_folder(p.ProjFileFolder);
    correct_folder(p.ObjFileFolder);
    if (p.ReconFileFolder.empty()) p.ReconFileFolder = p.ProjFileFolder;
}

// create_filename (hf_cpp_functions.hpp:117-135): <folder><root>_<n><suffix>
std::string numbered(const std::string& folder, const std::string& root, unsigned n, const std::string& suffix)
{
    return folder + root + "_" + std::to_string(n) + suffix;
}

long long file_bytes(const std::string& path)
{
    struct stat st;
    if (stat(path.c_str(), &st) != 0) return -1;
    return (long long)st.st_size;
}

recon_status_t read_floats(const std::string& path, float* dst, size_t n)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return fail(RECON_ERR_FILE_NOT_FOUND, "cannot open " + path);
    size_t got = std::fread(dst, sizeof(float), n, f);
    std::fclose(f);
    if (got != n) return fail(RECON_ERR_IO, "short read from " + path);
    return RECON_OK;
}

recon_status_t write_floats(const std::string& path, const float* src, size_t n)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return fail(RECON_ERR_IO, "cannot create " + path + ": " + std::strerror(errno));
    size_t put = std::fwrite(src, sizeof(float), n, f);
    int rc = std::fclose(f);
    if (put != n || rc != 0) return fail(RECON_ERR_IO, "short write to " + path);
    return RECON_OK;
}

// create_directory (hf_cpp_functions.hpp:198-231) without the prompt: an
// existing directory is accepted, a missing one is created (one level).
recon_status_t ensure_directory(const std::string& dir)
{
    if (dir.empty()) return RECON_OK;
    struct stat st;
    if (stat(dir.c_str(), &st) == 0) {
        if (S_ISDIR(st.st_mode)) return RECON_OK;
        return fail(RECON_ERR_IO, dir + " exists and is not a directory");
    }
    if (mkdir(dir.c_str(), 0755) != 0 && errno != EEXIST)
        return fail(RECON_ERR_IO, "cannot create directory " + dir + ": " + std::strerror(errno));
    return RECON_OK;
}

// check_projection_files (hf_cpp_functions.hpp:247-270)
recon_status_t check_projection_files(const recon_geometry_t& g, const Paths& p)
{
    const long long want = (long long)g.det.NumAxPixels * g.det.NumTAxPixels * 4;
    for (unsigned i = 0; i < g.scan.NumProj; ++i) {
        std::string f = numbered(p.ProjFileFolder, p.ProjFileNameRoot, i, p.ProjFileSuffix);
        long long b = file_bytes(f);
        if (b < 0) return fail(RECON_ERR_FILE_NOT_FOUND, "projection file does not exist: " + f);
        if (b != want)
            return fail(RECON_ERR_SIZE_MISMATCH, "projection file " + f + " has " + std::to_string(b) +
                                                     " bytes, the configuration implies " + std::to_string(want));
    }
    return RECON_OK;
}

// The .info parameter echo of WriteParameterFile (hf_siddon_class.hpp:
// 420-643): the configuration written back in the input file's format, so
// it can be read again as a configuration.
recon_status_t write_info(const std::string& path, const recon_geometry_t& g, const Paths& p)
{
    std::ofstream o(path.c_str());
    if (!o) return fail(RECON_ERR_IO, "cannot create " + path);
    o.setf(std::ios::fixed, std::ios::floatfield);
    o.precision(4);
    o << "# Calibration parameters\n";
    o << "R = " << g.cal.R << "\t# mm, source to detector\n";
    o << "Rf = " << g.cal.Rf << "\t# mm, source to rotation axis\n";
    o << "Ry = " << g.cal.Ry << "\t# mm, R + dy\n";
    o << "Dx = " << g.cal.Dx << "\t# mm, detector offset in x\n";
    o << "Dz = " << g.cal.Dz << "\t# mm, detector offset in z\n";
    o << "xangle = " << g.cal.xangle << "\t# rad, detector tilt about x\n";
    o << "yangle = " << g.cal.yangle << "\t# rad, detector tilt about y\n";
    o << "zangle = " << g.cal.zangle << "\t# rad, detector tilt about z\n";
    o << "M = " << g.cal.M << "\t# lens magnification\n\n";
    o << "# Detector parameters\n";
    o << "TAxPixels = " << g.det.NumTAxPixels << "\nAxPixels = " << g.det.NumAxPixels << "\n";
    o << "TAxPixDim = " << g.det.TAxPixDimMm << "\nAxPixDim = " << g.det.AxPixDimMm << "\n\n";
    o << "# Voxel volume parameters\n";
    o << "Xdim = " << g.vox.Xdim << "\nYdim = " << g.vox.Ydim << "\nZdim = " << g.vox.Zdim << "\n";
    o << "XVoxSize = " << g.vox.XVoxSize << "\nYVoxSize = " << g.vox.YVoxSize << "\nZVoxSize = " << g.vox.ZVoxSize
      << "\n\n";
    o << "# Scan parameters\n";
    o << "N_iteration = " << g.scan.N_iteration << "\nNumProj = " << g.scan.NumProj << "\nDeltaAng = "
      << g.scan.DeltaAng << "\n\n";
    o << "# File paths\n";
    o << "ProjFileFolder = " << p.ProjFileFolder << "\nProjFileNameRoot = " << p.ProjFileNameRoot
      << "\nProjFileSuffix = " << p.ProjFileSuffix << "\nReconFileFolder = " << p.ReconFileFolder
      << "\nReconFileNameRoot = " << p.ReconFileNameRoot << "\nReconFileSuffix = " << p.ReconFileSuffix << "\n\n";
    o << "ObjFileFolder = " << p.ObjFileFolder << "\nObjFileName = " << p.ObjFileName
      << "\nBpFileNameRoot = " << p.BpFileNameRoot << "\nBpFileSuffix = " << p.BpFileSuffix << "\n";
    if (!o) return fail(RECON_ERR_IO, "write failed: " + path);
    return RECON_OK;
}

struct Loaded {
    recon_geometry_t geom{};
    Paths paths;
    // optional resume keys (no reference counterpart): an image to start from
    // instead of f = 1, and the number of the first iteration to run
    std::string initial_volume;
    unsigned start_iteration = 0;
};

// m_check_files (hf_siddon_recon.hpp:196-226): configuration present, every
// key read, paths corrected.
recon_status_t load_config(const char* folder, const char* cfg, Loaded& L)
{
    if (!cfg) return fail(RECON_ERR_INVALID_ARGUMENT, "configuration file name is NULL");
    std::string dir = folder ? folder : "";
    correct_folder(dir);
    std::map<std::string, std::string> kv;
    RB_TRY(parse_config(dir + cfg, kv));
    RB_TRY(load_geometry(kv, L.geom));
    RB_TRY(load_paths(kv, L.paths));
    correct_paths(L.paths);
    if (kv.count("InitialVolume")) L.initial_volume = kv.at("InitialVolume");
    if (kv.count("StartIteration")) RB_TRY(get_number(kv, "StartIteration", L.start_iteration));
    return RECON_OK;
}

struct DevBuf {
    float* p = nullptr;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
    recon_status_t alloc(size_t n)
    {
        if (cudaMalloc(&p, n * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            return fail(RECON_ERR_OUT_OF_MEMORY, "device allocation failed");
        }
        return RECON_OK;
    }
};

struct PlanGuard {
    recon_plan_t p = nullptr;
    ~PlanGuard()
    {
        if (p) recon_plan_destroy(p);
    }
};

recon_status_t to_host(float* dst, const float* src, size_t n)
{
    cudaError_t e = cudaMemcpy(dst, src, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(RECON_ERR_CUDA, std::string("device to host copy: ") + cudaGetErrorString(e));
    }
    return RECON_OK;
}
recon_status_t to_device(float* dst, const float* src, size_t n)
{
    cudaError_t e = cudaMemcpy(dst, src, n * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(RECON_ERR_CUDA, std::string("host to device copy: ") + cudaGetErrorString(e));
    }
    return RECON_OK;
}

}  // namespace

extern "C" {

recon_status_t recon_geometry_from_cfg(const char* cfg_path, recon_geometry_t* geom, recon_filepaths_t* paths)
{
    if (!cfg_path || !geom) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    std::map<std::string, std::string> kv;
    RB_TRY(parse_config(cfg_path, kv));
    recon_geometry_t g{};
    RB_TRY(load_geometry(kv, g));
    if (paths) {
        Paths p;
        RB_TRY(load_paths(kv, p));
        RB_TRY(copy_path(p.ProjFileFolder, paths->ProjFileFolder, "ProjFileFolder"));
        RB_TRY(copy_path(p.ProjFileNameRoot, paths->ProjFileNameRoot, "ProjFileNameRoot"));
        RB_TRY(copy_path(p.ProjFileSuffix, paths->ProjFileSuffix, "ProjFileSuffix"));
        RB_TRY(copy_path(p.ReconFileFolder, paths->ReconFileFolder, "ReconFileFolder"));
        RB_TRY(copy_path(p.ReconFileNameRoot, paths->ReconFileNameRoot, "ReconFileNameRoot"));
        RB_TRY(copy_path(p.ReconFileSuffix, paths->ReconFileSuffix, "ReconFileSuffix"));
        RB_TRY(copy_path(p.ObjFileFolder, paths->ObjFileFolder, "ObjFileFolder"));
        RB_TRY(copy_path(p.ObjFileName, paths->ObjFileName, "ObjFileName"));
        RB_TRY(copy_path(p.BpFileNameRoot, paths->BpFileNameRoot, "BpFileNameRoot"));
        RB_TRY(copy_path(p.BpFileSuffix, paths->BpFileSuffix, "BpFileSuffix"));
    }
    *geom = g;
    return RECON_OK;
}

recon_status_t recon_mlem_from_cfg(const char* folder, const char* cfg, const recon_options_t* opt)
{
    Loaded L;
    RB_TRY(load_config(folder, cfg, L));
    RB_TRY(check_projection_files(L.geom, L.paths));  // m_check_reconstruction (hf_siddon_recon.hpp:294-313)
    const recon_geometry_t& g = L.geom;
    const size_t npix = (size_t)g.det.NumAxPixels * g.det.NumTAxPixels;
    const size_t nvox = (size_t)g.vox.Xdim * g.vox.Ydim * g.vox.Zdim;
    PlanGuard plan;
    RB_TRY(recon_plan_create(&g, opt, &plan.p));
    // the measured projections are read once (the reference re-reads every
    // view from disk in every iteration, hf_siddon_recon.hpp:446-449)
    std::vector<float> host(npix * (size_t)g.scan.NumProj);
    for (unsigned n = 0; n < g.scan.NumProj; ++n)
        RB_TRY(read_floats(numbered(L.paths.ProjFileFolder, L.paths.ProjFileNameRoot, n, L.paths.ProjFileSuffix),
                           host.data() + (size_t)n * npix, npix));
    DevBuf d_g, d_f;
    RB_TRY(d_g.alloc(host.size()));
    RB_TRY(d_f.alloc(nvox));
    RB_TRY(to_device(d_g.p, host.data(), host.size()));
    RB_TRY(recon_mlem_prepare(plan.p, nullptr));
    std::vector<float> f(nvox);
    if (L.initial_volume.empty()) {
        RB_TRY(recon_set_ones(d_f.p, nvox, nullptr));
    } else {
        // resume from a saved iterate (a written <ReconFileNameRoot>_<it> file)
        RB_TRY(read_floats(L.initial_volume, f.data(), nvox));
        RB_TRY(to_device(d_f.p, f.data(), nvox));
    }
    for (unsigned it = L.start_iteration; it < g.scan.N_iteration; ++it) {
        RB_TRY(recon_mlem_iteration(plan.p, d_g.p, d_f.p, nullptr));
        RB_TRY(to_host(f.data(), d_f.p, nvox));
        RB_TRY(write_floats(numbered(L.paths.ReconFileFolder, L.paths.ReconFileNameRoot, it, L.paths.ReconFileSuffix),
                            f.data(), nvox));
    }
    // a1_WriteReconParameters (hf_siddon_class.hpp:451-465)
    return write_info(L.paths.ReconFileFolder + L.paths.ReconFileNameRoot + ".info", g, L.paths);
}

recon_status_t recon_forward_projection_from_cfg(const char* folder, const char* cfg, const recon_options_t* opt)
{
    Loaded L;
    RB_TRY(load_config(folder, cfg, L));
    const recon_geometry_t& g = L.geom;
    const size_t npix = (size_t)g.det.NumAxPixels * g.det.NumTAxPixels;
    const size_t nvox = (size_t)g.vox.Xdim * g.vox.Ydim * g.vox.Zdim;
    // m_check_forward_projection (hf_siddon_recon.hpp:228-269)
    const std::string obj = L.paths.ObjFileFolder + L.paths.ObjFileName;
    long long b = file_bytes(obj);
    if (b < 0) return fail(RECON_ERR_FILE_NOT_FOUND, "object file does not exist: " + obj);
    if (b != (long long)(nvox * 4))
        return fail(RECON_ERR_SIZE_MISMATCH, "object file " + obj + " has " + std::to_string(b) +
                                                 " bytes, the configuration implies " + std::to_string(nvox * 4));
    RB_TRY(ensure_directory(L.paths.ProjFileFolder));
    std::vector<float> vol(nvox), img(npix);
    RB_TRY(read_floats(obj, vol.data(), nvox));
    PlanGuard plan;
    RB_TRY(recon_plan_create(&g, opt, &plan.p));
    DevBuf d_vol, d_img;
    RB_TRY(d_vol.alloc(nvox));
    RB_TRY(d_img.alloc(npix));
    RB_TRY(to_device(d_vol.p, vol.data(), nvox));
    for (unsigned n = 0; n < g.scan.NumProj; ++n) {  // m_forward_projection (:515-544)
        RB_TRY(recon_fp_views(plan.p, d_vol.p, n, 1, d_img.p, nullptr));
        RB_TRY(to_host(img.data(), d_img.p, npix));
        RB_TRY(write_floats(numbered(L.paths.ProjFileFolder, L.paths.ProjFileNameRoot, n, L.paths.ProjFileSuffix),
                            img.data(), npix));
    }
    return write_info(L.paths.ProjFileFolder + L.paths.ProjFileNameRoot + ".info", g, L.paths);
}

recon_status_t recon_backward_projection_from_cfg(const char* folder, const char* cfg, int write_per_angle,
                                                  const recon_options_t* opt)
{
    Loaded L;
    RB_TRY(load_config(folder, cfg, L));
    RB_TRY(check_projection_files(L.geom, L.paths));  // m_check_backward_projection (:271-292)
    const recon_geometry_t& g = L.geom;
    const size_t npix = (size_t)g.det.NumAxPixels * g.det.NumTAxPixels;
    const size_t nvox = (size_t)g.vox.Xdim * g.vox.Ydim * g.vox.Zdim;
    PlanGuard plan;
    RB_TRY(recon_plan_create(&g, opt, &plan.p));
    DevBuf d_img, d_view, d_total;
    RB_TRY(d_img.alloc(npix));
    RB_TRY(d_view.alloc(nvox));
    RB_TRY(d_total.alloc(nvox));
    if (cudaMemset(d_total.p, 0, nvox * sizeof(float)) != cudaSuccess)
        return fail(RECON_ERR_CUDA, "cudaMemset failed");
    std::vector<float> img(npix), vol(nvox);
    for (unsigned n = 0; n < g.scan.NumProj; ++n) {  // m_backward_projection (:546-592)
        RB_TRY(read_floats(numbered(L.paths.ProjFileFolder, L.paths.ProjFileNameRoot, n, L.paths.ProjFileSuffix),
                           img.data(), npix));
        RB_TRY(to_device(d_img.p, img.data(), npix));
        RB_TRY(recon_bp_views(plan.p, d_img.p, n, 1, d_view.p, nullptr));
        RB_TRY(recon_add(d_total.p, d_view.p, nvox, nullptr));
        if (write_per_angle) {
            RB_TRY(to_host(vol.data(), d_view.p, nvox));
            RB_TRY(write_floats(numbered(L.paths.ProjFileFolder, L.paths.BpFileNameRoot, n, L.paths.BpFileSuffix),
                                vol.data(), nvox));
        }
    }
    RB_TRY(to_host(vol.data(), d_total.p, nvox));
    RB_TRY(write_floats(L.paths.ProjFileFolder + L.paths.BpFileNameRoot + L.paths.BpFileSuffix, vol.data(), nvox));
    return write_info(L.paths.ProjFileFolder + L.paths.BpFileNameRoot + ".info", g, L.paths);
}

}  // extern "C"
