// march.cu -- ray-marching forward projection through a sampled volume.
//
// The reference's texture forward projector forward_projection
// (hf_cuda_kernels.cuh:126-180) takes one detector image, one view angle and
// one depth y0 of the view's frame: each pixel's ray is followed to depth y0
// (x0 = (y0+Rf)·u_id/R, z0 = (y0+Rf)·v_id/R, hf_cuda_kernels.cuh:155-156),
// rotated into the volume (x' = x0·cos + y0·sin, y' = -x0·sin + y0·cos,
// :158-159), sampled with tex3D and added times distance_traveled
// (hf_cuda_kernels.cuh:78-81, the ray length per YVoxSize of depth).  Its 3D
// texture is set up by texture_helper3D (hf_texture_helper.hpp:99-178) with
// border addressing and point filtering; the kernel passes coordinates
// normalised by L = (Ydim-1)·YVoxSize for every axis (:161-163).  The
// reference defines no caller, so the loop over depths is not given there.
//
// Here one thread follows one ray through all its depths in registers:
//   REFERENCE: the kernel's arithmetic as written (pixel_iterate without
//     rounding, the misalignment matrix, __fdividef, the angle in radians with
//     the reference's M_PI and its sine and cosine from the device's sincosf,
//     hf_cuda_kernels.cuh:146-147),
//     depths at the texel centres of the normalised y coordinate,
//     y0 = L·((k + 1/2)/Ydim - 1/2) for k = 0..Ydim-1, and the texel a
//     normalised, point-filtered, border-addressed tex3D returns:
//     floor(coordinate·size) inside [0, 1), 0 outside.  The texel is computed
//     in FP32 from the coordinate, not by the texture unit.
//   GEOMETRIC: the same rays and angle sense, IEEE divisions, depths spanning
//     the volume's bounding circle (y0 = -r + (k + 1/2)·YVoxSize, r the half
//     diagonal of the xy extent), and trilinear interpolation at voxel
//     centres with zero outside the volume: a plane-sampled line integral.
// The image is overwritten with the sum over all depths.
#include "internal.h"

#include <cmath>

namespace rb {
namespace march {

struct MarchGeom {
    int X, Y, Z, Nu, Nv;
    float vox[3], P0[3];
    float R, Rf, Ry, Dx, Dz, M, du, dv;  // du, dv: pixel pitches in mm (before M)
    float RM[9];
    float L;        // (Ydim - 1) * YVoxSize
    int nplanes;    // depths y0 = y_first + k * y_step
    float y_first, y_step;
    float angle_deg;  // REFERENCE: the view angle, turned into sine and cosine on the device
};

template <int MODE>
__global__ void __launch_bounds__(128) march_fp_kernel(MarchGeom G, float c, float s, const float* __restrict__ vol,
                                                        float* __restrict__ img)
// c, s: cosine and sine of the view angle (GEOMETRIC; REFERENCE computes its own)
{
    const int u = blockIdx.x * 32 + threadIdx.x, v = blockIdx.y * 4 + threadIdx.y;
    if (u >= G.Nu || v >= G.Nv) return;
    // pixel_iterate (hf_cuda_kernels.cuh:83-87)
    const float pu = -((float)G.Nu - 1.0f) / 2.0f * G.du * G.M + (float)u * G.du * G.M;
    const float pv = -((float)G.Nv - 1.0f) / 2.0f * G.dv * G.M + (float)v * G.dv * G.M;
    // hf_cuda_kernels.cuh:140-141
    const float den = G.Ry + G.RM[3] * pu + G.RM[5] * pv;
    float u_id, v_id, w;
    if (MODE == RECON_VOXEL_REFERENCE) {
        u_id = __fdividef(G.R, den) * (G.RM[0] * pu + G.RM[2] * pv + G.Dx);
        v_id = __fdividef(G.R, den) * (G.RM[6] * pu + G.RM[8] * pv + G.Dz);
        w = __fdividef(sqrtf(v_id * v_id + u_id * u_id + G.R * G.R), G.R) * G.vox[1];
    } else {
        u_id = G.R / den * (G.RM[0] * pu + G.RM[2] * pv + G.Dx);
        v_id = G.R / den * (G.RM[6] * pu + G.RM[8] * pv + G.Dz);
        w = sqrtf(v_id * v_id + u_id * u_id + G.R * G.R) / G.R * G.y_step;
    }
    if (MODE == RECON_VOXEL_REFERENCE) {
        // sincosf(alpha_deg * (float)M_PI / 180.0f) with #define M_PI 3.1415927
        // (hf_cuda_kernels.cuh:23, 146-147)
        sincosf(G.angle_deg * 3.1415927f / 180.0f, &s, &c);
    }
    const size_t plane = (size_t)G.X * G.Y;
    float acc = 0.0f;
    for (int k = 0; k < G.nplanes; ++k) {
        const float y0 = fmaf((float)k, G.y_step, G.y_first);
        if (MODE == RECON_VOXEL_REFERENCE) {
            const float x0 = __fdividef((y0 + G.Rf) * u_id, G.R);
            const float z0 = __fdividef((y0 + G.Rf) * v_id, G.R);
            const float xn = __fdividef(x0 * c + y0 * s, G.L) + 0.5f;
            const float yn = __fdividef(-x0 * s + y0 * c, G.L) + 0.5f;
            const float zn = __fdividef(z0, G.L) + 0.5f;
            if (!(xn >= 0.0f && xn < 1.0f && yn >= 0.0f && yn < 1.0f && zn >= 0.0f && zn < 1.0f)) continue;
            const int ix = min((int)(xn * (float)G.X), G.X - 1);
            const int iy = min((int)(yn * (float)G.Y), G.Y - 1);
            const int iz = min((int)(zn * (float)G.Z), G.Z - 1);
            acc = acc + __ldg(vol + (size_t)ix + (size_t)iy * G.X + (size_t)iz * plane) * w;
        } else {
            const float d = (y0 + G.Rf) / G.R;
            const float x0 = d * u_id, z0 = d * v_id;
            const float xa = x0 * c + y0 * s, ya = -x0 * s + y0 * c;
            // voxel-centre coordinates: voxel i spans [i, i+1), its centre at i + 1/2
            const float fx = (xa - G.P0[0]) / G.vox[0] - 0.5f;
            const float fy = (ya - G.P0[1]) / G.vox[1] - 0.5f;
            const float fz = (z0 - G.P0[2]) / G.vox[2] - 0.5f;
            if (!(fx > -1.0f && fx < (float)G.X && fy > -1.0f && fy < (float)G.Y && fz > -1.0f && fz < (float)G.Z))
                continue;
            const float gx = floorf(fx), gy = floorf(fy), gz = floorf(fz);
            const int ix = (int)gx, iy = (int)gy, iz = (int)gz;
            const float ax = fx - gx, ay = fy - gy, az = fz - gz;
            float sample = 0.0f;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const int jx = ix + (t & 1), jy = iy + ((t >> 1) & 1), jz = iz + (t >> 2);
                if (jx < 0 || jx >= G.X || jy < 0 || jy >= G.Y || jz < 0 || jz >= G.Z) continue;
                const float wt = ((t & 1) ? ax : 1.0f - ax) * (((t >> 1) & 1) ? ay : 1.0f - ay) *
                                 ((t >> 2) ? az : 1.0f - az);
                sample = fmaf(wt, __ldg(vol + (size_t)jx + (size_t)jy * G.X + (size_t)jz * plane), sample);
            }
            acc = fmaf(sample, w, acc);
        }
    }
    img[(size_t)u + (size_t)v * G.Nu] = acc;
}

}  // namespace march

recon_status_t march_fp_view(Plan& P, const float* vol, float angle_deg, int mode, float* img, cudaStream_t s)
{
    const recon_geometry_t& g = P.geom;
    march::MarchGeom G;
    G.X = (int)g.vox.Xdim;
    G.Y = (int)g.vox.Ydim;
    G.Z = (int)g.vox.Zdim;
    G.Nu = (int)g.det.NumAxPixels;
    G.Nv = (int)g.det.NumTAxPixels;
    G.vox[0] = g.vox.XVoxSize;
    G.vox[1] = g.vox.YVoxSize;
    G.vox[2] = g.vox.ZVoxSize;
    G.P0[0] = (float)(-(double)G.X / 2.0 * G.vox[0]);
    G.P0[1] = (float)(-(double)G.Y / 2.0 * G.vox[1]);
    G.P0[2] = (float)(-(double)G.Z / 2.0 * G.vox[2]);
    G.R = g.cal.R;
    G.Rf = g.cal.Rf;
    G.Ry = g.cal.Ry;
    G.Dx = g.cal.Dx;
    G.Dz = g.cal.Dz;
    G.M = g.cal.M;
    G.du = g.det.AxPixDimMm;
    G.dv = g.det.TAxPixDimMm;
    for (int i = 0; i < 9; ++i) G.RM[i] = P.RM[i];
    G.L = ((float)G.Y - 1.0f) * G.vox[1];
    G.angle_deg = angle_deg;
    float c, sn;
    if (mode == RECON_VOXEL_REFERENCE) {
        G.nplanes = G.Y;
        G.y_step = G.L / (float)G.Y;
        G.y_first = G.L * (0.5f / (float)G.Y - 0.5f);
        sn = c = 0.0f;  // the kernel takes sincosf of angle_deg itself
    } else {
        const double hx = 0.5 * G.X * G.vox[0], hy = 0.5 * G.Y * G.vox[1];
        const double r = std::sqrt(hx * hx + hy * hy);
        G.y_step = G.vox[1];
        G.nplanes = (int)std::ceil(2.0 * r / G.y_step);
        G.y_first = (float)(-r + 0.5 * G.y_step);
        const double a = (double)angle_deg / 180.0;
        c = (float)std::cos(M_PI * a);
        sn = (float)std::sin(M_PI * a);
    }
    const dim3 blk(32, 4), grid((G.Nu + 31) / 32, (G.Nv + 3) / 4);
    if (mode == RECON_VOXEL_REFERENCE)
        march::march_fp_kernel<RECON_VOXEL_REFERENCE><<<grid, blk, 0, s>>>(G, c, sn, vol, img);
    else
        march::march_fp_kernel<RECON_VOXEL_GEOMETRIC><<<grid, blk, 0, s>>>(G, c, sn, vol, img);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

}  // namespace rb
