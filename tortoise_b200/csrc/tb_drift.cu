// tb_drift.cu -- field-driven drift: the DG upwind Vlasov operator of the
// reference (include/Physics/Transport/Vlasov.hpp:69-118), as a block-sparse
// operator with 3x3 blocks (self plus up to three face neighbours) evaluated
// matrix-free: one thread per element reads its own 3 coefficients and those
// of the upwind neighbours, and adds (volume - surface) into the pre-M^-1
// accumulator (M^-1 is applied with the collision terms).
//
// Geometry follows Mesh<2>: periodic adjacency and faces (src/Geometry/
// Structured/DirectSpace/Mesh.cpp:573-660); basis derivatives evaluated on
// calculate_verticesCoord (Mesh.cpp:147-163, 222-241), which places vertices
// at relativeOrigin + dGVec * (section + vertex).
#include "tb_dp45.cuh"
#include "tb_kernels.cuh"

namespace tb {

__device__ __forceinline__ int adjacent_element(int nx, int nt, int e, int face) {
    if (e & 1) {
        if (face == 0) return (e + 2 * nx - 1 + nt) % nt;
        if (face == 1) return e - 1;
        return ((e - 1) % (2 * nx) == 0) ? e + 2 * nx - 3 : e - 3;
    } else {
        if (face == 0) return ((e + 2) % (2 * nx) == 0) ? e - 2 * nx + 3 : e + 3;
        if (face == 1) return e + 1;
        return (e - 2 * nx + 1 + nt) % nt;
    }
}

__device__ __forceinline__ void face_normal(const MeshDev& m, int e, int face, double n[2]) {
    const double d00 = m.dG[0][0], d01 = m.dG[0][1], d10 = m.dG[1][0], d11 = m.dG[1][1];
    double v0, v1, sgn;
    if (e & 1) {
        if (face == 0) { v0 = d10; v1 = -d00; sgn = (v0 * d01 + v1 * d11 > 0.) ? 1. : -1.; }
        else if (face == 1) { v0 = d11 + d10; v1 = -d01 - d00; sgn = (v0 * d00 + v1 * d10 > 0.) ? 1. : -1.; }
        else { v0 = d11; v1 = -d01; sgn = (v0 * d00 + v1 * d10 > 0.) ? -1. : 1.; }
    } else {
        if (face == 0) { v0 = d11; v1 = -d01; sgn = (v0 * d00 + v1 * d10 > 0.) ? 1. : -1.; }
        else if (face == 1) { v0 = d11 + d10; v1 = -d01 - d00; sgn = (v0 * d00 + v1 * d10 > 0.) ? -1. : 1.; }
        else { v0 = d10; v1 = -d00; sgn = (v0 * d01 + v1 * d11 > 0.) ? -1. : 1.; }
    }
    const double nn = sqrt(v0 * v0 + v1 * v1);
    n[0] = v0 / nn * sgn;
    n[1] = v1 / nn * sgn;
}

__device__ __forceinline__ double face_area(const MeshDev& m, int e, int face) {
    const double d00 = m.dG[0][0], d01 = m.dG[0][1], d10 = m.dG[1][0], d11 = m.dG[1][1];
    const int f = (e & 1) ? face : 2 - face;   // odd: 0->col0 1->diag 2->col1; even mirrored
    if (f == 0) return sqrt(d00 * d00 + d10 * d10);
    if (f == 1) return sqrt((d00 + d01) * (d00 + d01) + (d10 + d11) * (d10 + d11));
    return sqrt(d01 * d01 + d11 * d11);
}

// gaussPointsSide<2,2> (Vlasov.hpp:49-62)
__device__ __forceinline__ void side_point(int side, int q, double& x, double& y) {
    const double g = q ? TB_GP1_1 : TB_GP1_0;
    if (side == 0) { x = 1. - g; y = g; }
    else if (side == 1) { x = 0.; y = g; }
    else { x = g; y = 0.; }
}

__global__ void __launch_bounds__(256) k_drift(ElemDev ed, const double* __restrict__ f, double* __restrict__ acc,
                                               const DPCtl* __restrict__ ctl) {
    const int band = ed.blk_band[blockIdx.x];
    const BandDev& bd = ed.bands[band];
    const double vel0 = bd.vel[0], vel1 = bd.vel[1];
    if (vel0 == 0.0 && vel1 == 0.0) return;
    if (ctl && ctl[ed.band_run[band]].done) return;
    const int e = (blockIdx.x - ed.blk_first[band]) * blockDim.x + threadIdx.x;
    if (e >= bd.ne) return;
    const MeshDev m = bd.mesh;
    const double gpa = TB_GP2_A, gpb = TB_GP2_B, gw = TB_GW2;
    const double gx[3] = {gpa, gpb, gpa}, gy[3] = {gpa, gpa, gpb};
    const double* fb = f + bd.off;
    const int nt = m.ne;
    const double c0 = fb[3 * e], c1 = fb[3 * e + 1], c2 = fb[3 * e + 2];
    // volumeFlux (Vlasov.hpp:78-92)
    double gi = 0.0;
#pragma unroll
    for (int q = 0; q < 3; ++q) gi += ((c1 * gx[q] + c2 * gy[q]) + c0) * gw;
    const int s = e / 2, par = e & 1;
    const double sx = double(s % m.nx), sy = double(s / m.nx);
    double vx[3], vy[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double ox = (k == 0) ? 0.0 : (par ? (k == 1 ? 0.0 : 1.0) : 1.0);
        const double oy = (k == 0) ? 0.0 : (par ? 1.0 : (k == 1 ? 0.0 : 1.0));
        const double px = sx + ox, py = sy + oy;
        vx[k] = m.rel_origin[0] + (m.dG[0][0] * px + m.dG[0][1] * py);
        vy[k] = m.rel_origin[1] + (m.dG[1][0] * px + m.dG[1][1] * py);
    }
    const double v0X = vx[0], v0Y = vy[0], v1X = vx[1], v1Y = vy[1], v2X = vx[2], v2Y = vy[2];
    const double denx = v0Y * (v1X - v2X) + v1Y * (v2X - v0X) + v2Y * (v0X - v1X);
    const double deny = v0X * (v1Y - v2Y) + v1X * (v2Y - v0Y) + v2X * (v0Y - v1Y);
    const double dx[3] = {0.0, (v0Y - v2Y) / denx, -(v0Y - v1Y) / denx};
    const double dy[3] = {0.0, (v0X - v2X) / deny, -(v0X - v1X) / deny};
    double vol[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int bb = 0; bb < 3; ++bb) vol[bb] += m.vol * vel0 * (dx[bb] * gi);
#pragma unroll
    for (int bb = 0; bb < 3; ++bb) vol[bb] += m.vol * vel1 * (dy[bb] * gi);
    // surfaceFlux (Vlasov.hpp:94-118), upwind by the sign of v.n
    double sur[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int side = 0; side < 3; ++side) {
        double n[2];
        face_normal(m, e, side, n);
        const double sv = vel0 * n[0] + vel1 * n[1];
        int ei, si;
        if (sv > 0.) { ei = e; si = side; }
        else { ei = adjacent_element(m.nx, nt, e, side); si = 2 - side; }
        const double f0 = fb[3 * ei], f1 = fb[3 * ei + 1], f2 = fb[3 * ei + 2];
        const double area = face_area(m, e, side);
        double fv[2], bx[2], by[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            double xi, yi;
            side_point(si, q, xi, yi);
            fv[q] = (f1 * xi + f2 * yi) + f0;
            side_point(side, q, bx[q], by[q]);
        }
#pragma unroll
        for (int bb = 0; bb < 3; ++bb) {
            double a = 0.0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const double phi = (bb == 0) ? 1.0 : (bb == 1 ? bx[q] : by[q]);
                a += phi * fv[q] * 0.5;
            }
            sur[bb] += sv * a * area;
        }
    }
    double* o = acc + bd.off + 3 * (int64_t)e;
#pragma unroll
    for (int bb = 0; bb < 3; ++bb) o[bb] += vol[bb] - sur[bb];
}

int launch_drift(const ElemDev& ed, const double* f, double* acc, const DPCtl* ctl, cudaStream_t s) {
    k_drift<<<ed.nblk, 256, 0, s>>>(ed, f, acc, ctl);
    TB_CUDA(cudaGetLastError());
    return TB_OK;
}

}  // namespace tb
