// hype_io.cu -- the reference's file formats, written from (and read into)
// the device-resident state of a solver:
//   restart files  PETSc binary Vec of the conserved state, as
//                  PetscViewerBinaryOpen + VecView(U) writes restart1/2.bin
//                  (post_process.c:47-64) and VecLoad reads it (hype.c:316-325);
//   solution files VTK XML structured grid of the primitive variables, as
//                  PetscViewerVTKOpen + DMView + VecView(Ctx->W) writes
//                  sol-%08d.vts (post_process.c:25-45, hype.c:388-399), the
//                  files HyPE-2D/plot.py reads.
// The primitive variables come from a device kernel that applies the same
// PDECons2Prim as the stage kernels (ComputePrimitiveVariables,
// post_process.c:165-200).  Built with --fmad=false.
#include <cuda_runtime.h>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/hype_gpu.h"
#include "hype_internal.h"

namespace hype {

template <int SYS>
__global__ void cons2prim_kernel(const double *__restrict__ planes, double *__restrict__ prim, int nx, int ny, int pitch,
                                 long long plane, Eos eos)
{
    using S = System<SYS>;
    const long long n = (long long)nx * ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const long long gi = (k / nx) * pitch + k % nx;
        double Q[S::NV], V[S::NV];
#pragma unroll
        for (int c = 0; c < S::NV; ++c) Q[c] = planes[c * plane + gi];
        S::cons2prim(eos, Q, V);
#pragma unroll
        for (int c = 0; c < S::NV; ++c) prim[k * S::NV + c] = V[c];
    }
}

cudaError_t launch_cons2prim(int sys, const Eos &eos, const double *planes, double *prim_aos, int nx, int ny, int pitch,
                             long long plane, cudaStream_t s)
{
    const long long n = (long long)nx * ny;
    const unsigned blocks = (unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    switch (sys) {
    case SYS_EULER: cons2prim_kernel<SYS_EULER><<<blocks, 256, 0, s>>>(planes, prim_aos, nx, ny, pitch, plane, eos); break;
    case SYS_KAPILA: cons2prim_kernel<SYS_KAPILA><<<blocks, 256, 0, s>>>(planes, prim_aos, nx, ny, pitch, plane, eos); break;
    default: cons2prim_kernel<SYS_BN><<<blocks, 256, 0, s>>>(planes, prim_aos, nx, ny, pitch, plane, eos); break;
    }
    return cudaGetLastError();
}

}  // namespace hype

using namespace hype;

namespace {

// PETSc binary files are big-endian
void put_be32(std::vector<unsigned char> &b, int v)
{
    const unsigned u = (unsigned)v;
    for (int k = 3; k >= 0; --k) b.push_back((unsigned char)(u >> (8 * k)));
}
void put_be64(unsigned char *p, double d)
{
    unsigned long long u;
    std::memcpy(&u, &d, 8);
    for (int k = 7; k >= 0; --k) *p++ = (unsigned char)(u >> (8 * k));
}
double get_be64(const unsigned char *p)
{
    unsigned long long u = 0;
    for (int k = 0; k < 8; ++k) u = (u << 8) | p[k];
    double d;
    std::memcpy(&d, &u, 8);
    return d;
}
int get_be32(const unsigned char *p)
{
    return (int)(((unsigned)p[0] << 24) | ((unsigned)p[1] << 16) | ((unsigned)p[2] << 8) | (unsigned)p[3]);
}

constexpr int VEC_FILE_CLASSID = 1211214;   // PETSc's class id of a Vec in a binary file

// field names of hype.c:141-174 (DMDASetFieldName), in component order
const char *const kFieldNames[3][9] = {
    {"density", "x-velocity", "y-velocity", "pressure"},
    {"density1", "density2", "x-velocity", "y-velocity", "pressure", "phi"},
    {"density_s", "x-velocity_s", "y-velocity_s", "pressure_s", "density_g", "x-velocity_g", "y-velocity_g", "pressure_g",
     "phi_s"},
};

}  // namespace

extern "C" {

int hype_write_restart(hype_solver *s, const char *path)
{
    if (!s || !path) return HYPE_ERR_INVALID;
    hype_config c;
    int rc = hype_solver_config(s, &c);
    if (rc) return rc;
    const int nv = hype_nvar(c.system);
    const size_t n = (size_t)c.nx * c.ny * nv;
    std::vector<double> U(n);
    if ((rc = hype_get_state(s, U.data()))) return rc;
    std::vector<unsigned char> head;
    put_be32(head, VEC_FILE_CLASSID);
    put_be32(head, (int)n);
    std::vector<unsigned char> body(n * 8);
    for (size_t k = 0; k < n; ++k) put_be64(&body[k * 8], U[k]);
    FILE *f = std::fopen(path, "wb");
    if (!f) return HYPE_ERR_INVALID;
    const bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size() && std::fwrite(body.data(), 1, body.size(), f) == body.size();
    std::fclose(f);
    if (!ok) return HYPE_ERR_INVALID;
    // the viewer's companion file: the Vec's block size (the DMDA's dof)
    const std::string info = std::string(path) + ".info";
    FILE *fi = std::fopen(info.c_str(), "w");
    if (fi) {
        std::fprintf(fi, "-vecload_block_size %d\n", nv);
        std::fclose(fi);
    }
    return HYPE_OK;
}

int hype_read_restart(hype_solver *s, const char *path)
{
    if (!s || !path) return HYPE_ERR_INVALID;
    hype_config c;
    int rc = hype_solver_config(s, &c);
    if (rc) return rc;
    const size_t n = (size_t)c.nx * c.ny * hype_nvar(c.system);
    FILE *f = std::fopen(path, "rb");
    if (!f) return HYPE_ERR_INVALID;
    unsigned char head[8];
    std::vector<unsigned char> body(n * 8);
    const bool ok = std::fread(head, 1, 8, f) == 8 && get_be32(head) == VEC_FILE_CLASSID && get_be32(head + 4) == (int)n &&
                    std::fread(body.data(), 1, body.size(), f) == body.size();
    std::fclose(f);
    if (!ok) return HYPE_ERR_INVALID;
    std::vector<double> U(n);
    for (size_t k = 0; k < n; ++k) U[k] = get_be64(&body[k * 8]);
    return hype_set_state(s, U.data());
}

int hype_write_vts(hype_solver *s, const char *path)
{
    if (!s || !path) return HYPE_ERR_INVALID;
    hype_config c;
    int rc = hype_solver_config(s, &c);
    if (rc) return rc;
    const int nv = hype_nvar(c.system);
    const size_t ncell = (size_t)c.nx * c.ny;
    std::vector<double> W(ncell * nv);
    if ((rc = hype_get_primitive(s, W.data()))) return rc;
    // DMDASetUniformCoordinates(x_min + h/2, x_max + h/2, ...) (hype.c:132-135):
    // spacing (max - min)/N on a periodic axis, (max - min)/(N - 1) otherwise
    const double h = (c.x_max - c.x_min) / (double)c.nx;
    const bool px = c.bc_left == HYPE_BC_PERIODIC, py = c.bc_bottom == HYPE_BC_PERIODIC;
    const double x0 = c.x_min + 0.5 * h, x1 = c.x_max + 0.5 * h;
    const double y0 = c.y_min + 0.5 * h, y1 = c.y_max + 0.5 * h;
    const double hx = (x1 - x0) / (double)(px ? c.nx : c.nx - 1);
    const double hy = (y1 - y0) / (double)(py ? c.ny : c.ny - 1);
    FILE *f = std::fopen(path, "wb");
    if (!f) return HYPE_ERR_INVALID;
    const unsigned long long pts_bytes = 3ull * ncell * 8, fld_bytes = (unsigned long long)ncell * 8;
    std::fprintf(f, "<?xml version=\"1.0\"?>\n");
    std::fprintf(f, "<VTKFile type=\"StructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n");
    std::fprintf(f, "  <StructuredGrid WholeExtent=\"0 %d 0 %d 0 0\">\n", c.nx - 1, c.ny - 1);
    std::fprintf(f, "    <Piece Extent=\"0 %d 0 %d 0 0\">\n", c.nx - 1, c.ny - 1);
    unsigned long long off = 0;
    std::fprintf(f, "      <Points>\n        <DataArray type=\"Float64\" Name=\"Position\" NumberOfComponents=\"3\" format=\"appended\" offset=\"%llu\" />\n      </Points>\n", off);
    off += 8 + pts_bytes;
    std::fprintf(f, "      <PointData Scalars=\"ScalarPointData\">\n");
    for (int q = 0; q < nv; ++q) {
        std::fprintf(f, "        <DataArray type=\"Float64\" Name=\"sol.%s\" NumberOfComponents=\"1\" format=\"appended\" offset=\"%llu\" />\n",
                     kFieldNames[c.system][q], off);
        off += 8 + fld_bytes;
    }
    std::fprintf(f, "      </PointData>\n    </Piece>\n  </StructuredGrid>\n  <AppendedData encoding=\"raw\">\n_");
    bool ok = std::fwrite(&pts_bytes, 8, 1, f) == 1;
    std::vector<double> buf(3 * (size_t)c.nx);
    for (int j = 0; j < c.ny && ok; ++j) {
        for (int i = 0; i < c.nx; ++i) {
            buf[3 * i] = x0 + hx * i;
            buf[3 * i + 1] = y0 + hy * j;
            buf[3 * i + 2] = 0.0;
        }
        ok = std::fwrite(buf.data(), 8, buf.size(), f) == buf.size();
    }
    std::vector<double> col(ncell);
    for (int q = 0; q < nv && ok; ++q) {
        for (size_t k = 0; k < ncell; ++k) col[k] = W[k * nv + q];
        ok = std::fwrite(&fld_bytes, 8, 1, f) == 1 && std::fwrite(col.data(), 8, ncell, f) == ncell;
    }
    std::fprintf(f, "\n  </AppendedData>\n</VTKFile>\n");
    std::fclose(f);
    return ok ? HYPE_OK : HYPE_ERR_INVALID;
}

// The output schedule of MonitorFunction (post_process.c:12-64), called by TS
// before the first step (step 0) and after every step, and the final solution
// file of hype.c:386-399.
static int monitor_outputs(hype_solver *s, int step, int write_interval, int restart_interval, const std::string &dir)
{
    int rc = HYPE_OK;
    char name[64];
    if (write_interval != 0 && step % write_interval == 0) {
        std::snprintf(name, sizeof(name), "sol-%08d.vts", step);
        if ((rc = hype_write_vts(s, (dir + name).c_str()))) return rc;
    }
    if (restart_interval != 0) {
        if (step % restart_interval == 0 && (rc = hype_write_restart(s, (dir + "restart1.bin").c_str()))) return rc;
        if ((step + 7) % restart_interval == 0 && (rc = hype_write_restart(s, (dir + "restart2.bin").c_str()))) return rc;
    }
    return rc;
}

int hype_solve_monitored(hype_solver *s, double t0, double t_final, int max_steps, int write_interval, int restart_interval,
                         const char *dir, int *steps_done, double *t_end, double *dt_next)
{
    if (!s || max_steps < 0 || write_interval < 0 || restart_interval < 0) return HYPE_ERR_INVALID;
    std::string d = dir ? dir : "";
    if (!d.empty() && d.back() != '/') d += '/';
    int rc = hype_begin(s, t0, t_final, max_steps);
    if (rc) return rc;
    int step = 0, steps = 0;
    double t = t0, dtn = 0.0;
    if ((rc = monitor_outputs(s, 0, write_interval, restart_interval, d))) return rc;
    while (step < max_steps) {
        // run up to the next step that writes something (or the end)
        int next = max_steps;
        for (int k = step + 1; k < max_steps; ++k)
            if ((write_interval && k % write_interval == 0) ||
                (restart_interval && (k % restart_interval == 0 || (k + 7) % restart_interval == 0))) { next = k; break; }
        if ((rc = hype_advance(s, next - step))) return rc;
        rc = hype_wait(s, &steps, &t, &dtn);
        if (rc) return rc;
        const bool stopped = steps < next;   // t_final reached on the way
        if (steps > step && (rc = monitor_outputs(s, steps, write_interval, restart_interval, d))) return rc;
        step = steps;
        if (stopped) break;
    }
    char name[64];
    std::snprintf(name, sizeof(name), "sol-%08d.vts", steps);   // hype.c:392-399
    if ((rc = hype_write_vts(s, (d + name).c_str()))) return rc;
    if (steps_done) *steps_done = steps;
    if (t_end) *t_end = t;
    if (dt_next) *dt_next = dtn;
    return HYPE_OK;
}

}  // extern "C"
