// mps_vtk.cu -- VTK rectilinear-grid output straight from device buffers.
//
// The reference writes its solution arrays as VTK XML RectilinearGrid files
// with raw appended Float64 data (mgridlib/cartwrite.f90): one serial .vtr
// (Writeserialvtrfile, :8-161), one .vtr piece per rank (Writevtrfile,
// :163-317) and the .pvtr index of the pieces (Writepvtrfile, :319-438).
// The files here carry the same bytes: the same XML lines and attribute
// formatting (offsets and extents as right-justified 8-character integers,
// as Fortran's (i8) edit descriptor writes them), the same appended block
// layout (a 4-byte size, then the cell values in Fortran order, i fastest),
// the same node coordinates off + (i-1) * len/l.
//
// The cell data come from ghosted device arrays: a kernel gathers the
// interior of one field into a contiguous device buffer, one
// cudaMemcpyAsync brings it into one of two pinned host buffers, and the
// file write of a field overlaps the gather and copy of the next.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <sys/types.h>
#include <vector>

#include "../../include/mps_linsolve.h"

namespace {

constexpr int VTPB = 256;

// interior (lx, ly, lz) of a ghosted (lx+2)(ly+2)(lz+2) Fortran-order field
__global__ void __launch_bounds__(VTPB) k_interior(int lx, int ly, int lz, const double* __restrict__ g,
                                                  double* __restrict__ out)
{
    const long long n = (long long)lx * ly * lz;
    const long long t = (long long)blockIdx.x * VTPB + threadIdx.x;
    if (t >= n) return;
    const int i = (int)(t % lx);
    const long long r = t / lx;
    const int j = (int)(r % ly);
    const int k = (int)(r / ly);
    out[t] = __ldg(&g[(i + 1) + (long long)(lx + 2) * ((j + 1) + (long long)(ly + 2) * (k + 1))]);
}

// Fortran (i8): right-justified in 8 characters
std::string i8(long long v)
{
    char b[32];
    std::snprintf(b, sizeof(b), "%8lld", v);
    return std::string(b);
}

// the extent string of cartwrite.f90 (:78-79): the six (i8) fields joined by
// single blanks, except that ymax and zmin are concatenated directly (their
// separation is zmin's own leading blanks)
std::string extent(long long x0, long long x1, long long y0, long long y1, long long z0, long long z1)
{
    return i8(x0) + " " + i8(x1) + " " + i8(y0) + " " + i8(y1) + i8(z0) + " " + i8(z1);
}

struct File {
    FILE* f = nullptr;
    bool ok = true;
    explicit File(const std::string& path) { f = std::fopen(path.c_str(), "wb"); ok = f != nullptr; }
    ~File()
    {
        if (f) std::fclose(f);
    }
    void put(const std::string& s)
    {
        if (ok && std::fwrite(s.data(), 1, s.size(), f) != s.size()) ok = false;
    }
    void put(const void* p, size_t n)
    {
        if (ok && n && std::fwrite(p, 1, n, f) != n) ok = false;
    }
    void put_i32(int v) { put(&v, sizeof(int)); }
};

// a name as Fortran's trim() leaves it: trailing blanks dropped
std::string rtrim(const char* s)
{
    std::string r(s);
    while (!r.empty() && r.back() == ' ') r.pop_back();
    return r;
}

bool names_ok(int n, const char* const* names)
{
    if (n < 0 || (n > 0 && !names)) return false;
    for (int i = 0; i < n; i++)
        if (!names[i]) return false;
    return true;
}

// one .vtr: header, cell-data and coordinate arrays, appended raw data
int write_vtr(const std::string& path, const std::string& whole, const std::string& piece, int lx, int ly, int lz,
              const double off[3], const double len[3], int nscalars, const char* const* names,
              const double* const* fields, cudaStream_t s)
{
    const long long ncell = (long long)lx * ly * lz;
    const int scalars_size = (int)(ncell * 8);
    File F(path);
    if (!F.ok) return MPS_ERR_BAD_ARG;
    const char nl = '\n';
    F.put(std::string("<?xml version=\"1.0\"?>") + nl);
    F.put(std::string("<VTKFile type=\"RectilinearGrid\" version=\"0.1\" byte_order=\"LittleEndian\">") + nl);
    F.put("  <RectilinearGrid WholeExtent=\"" + whole + "\">" + nl);
    F.put("    <Piece Extent=\"" + piece + "\">" + nl);
    F.put(std::string("      <PointData>  </PointData>") + nl);
    F.put(std::string("      <CellData> ") + nl);
    long long off_b = 0;
    for (int i = 0; i < nscalars; i++) {
        F.put("         <DataArray type=\"Float64\" Name=\"" + rtrim(names[i]) +
              "\" format=\"appended\" offset=\"" + i8(off_b) + "\"           />" + nl);
        off_b += 4 + scalars_size;
    }
    F.put(std::string("      </CellData>") + nl);
    F.put(std::string("      <Coordinates>") + nl);
    const int nn[3] = {lx + 1, ly + 1, lz + 1};
    const char* ax[3] = {"X", "Y", "Z"};
    for (int a = 0; a < 3; a++) {
        F.put(std::string("<DataArray type=\"Float64\" Name=\"") + ax[a] + "\"  format=\"appended\" offset=\"" +
              i8(off_b) + "\" />" + nl);
        off_b += 4 + 8LL * nn[a];
    }
    F.put(std::string("      </Coordinates>") + nl);
    F.put(std::string("    </Piece>") + nl);
    F.put(std::string("  </RectilinearGrid>") + nl);
    F.put(std::string("  <AppendedData encoding=\"raw\">") + nl);
    F.put("_");
    // cell data: gather -> pinned copy -> file, two stages in flight
    int st = MPS_OK;
    if (nscalars > 0) {
        double* dbuf = nullptr;
        double* hbuf[2] = {nullptr, nullptr};
        cudaEvent_t done[2] = {nullptr, nullptr};
        if (cudaMallocAsync((void**)&dbuf, sizeof(double) * ncell * 2, s) != cudaSuccess ||
            cudaMallocHost((void**)&hbuf[0], sizeof(double) * ncell) != cudaSuccess ||
            cudaMallocHost((void**)&hbuf[1], sizeof(double) * ncell) != cudaSuccess ||
            cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming) != cudaSuccess)
            st = MPS_ERR_CUDA;
        const unsigned nb = (unsigned)((ncell + VTPB - 1) / VTPB);
        auto issue = [&](int i) {
            const int b = i & 1;
            k_interior<<<nb, VTPB, 0, s>>>(lx, ly, lz, fields[i], dbuf + b * ncell);
            cudaMemcpyAsync(hbuf[b], dbuf + b * ncell, sizeof(double) * ncell, cudaMemcpyDeviceToHost, s);
            cudaEventRecord(done[b], s);
        };
        if (st == MPS_OK) issue(0);
        for (int i = 0; i < nscalars && st == MPS_OK; i++) {
            if (i + 1 < nscalars) issue(i + 1);
            if (cudaEventSynchronize(done[i & 1]) != cudaSuccess) {
                st = MPS_ERR_CUDA;
                break;
            }
            F.put_i32(scalars_size);
            F.put(hbuf[i & 1], sizeof(double) * ncell);
        }
        if (st == MPS_OK && cudaGetLastError() != cudaSuccess) st = MPS_ERR_CUDA;
        if (dbuf) cudaFreeAsync(dbuf, s);
        cudaStreamSynchronize(s);
        for (int b = 0; b < 2; b++) {
            if (hbuf[b]) cudaFreeHost(hbuf[b]);
            if (done[b]) cudaEventDestroy(done[b]);
        }
        if (st) return st;
    }
    for (int a = 0; a < 3; a++) {  // node coordinates off + (i-1) len/l (:57-67)
        const double d = len[a] / (nn[a] - 1);
        std::vector<double> c(nn[a]);
        for (int i = 0; i < nn[a]; i++) c[i] = off[a] + i * d;
        F.put_i32(nn[a] * 8);
        F.put(c.data(), sizeof(double) * c.size());
    }
    F.put(std::string(1, nl) + "  </AppendedData>" + nl);
    F.put(std::string("</VTKFile>") + nl);
    return F.ok ? MPS_OK : MPS_ERR_BAD_ARG;
}

}  // namespace

extern "C" {

int mps_write_vtr_dev(const char* filename, const mps_grid* g, const double off[3], int nscalars,
                      const char* const* names, const double* const* fields, void* stream)
{
    if (!filename || !g || g->lx < 1 || g->ly < 1 || g->lz < 1 || !names_ok(nscalars, names) ||
        (nscalars > 0 && !fields))
        return MPS_ERR_BAD_ARG;
    for (int i = 0; i < nscalars; i++)
        if (!fields[i]) return MPS_ERR_BAD_ARG;
    const double o[3] = {off ? off[0] : 0.0, off ? off[1] : 0.0, off ? off[2] : 0.0};
    const double len[3] = {g->llenx, g->lleny, g->llenz};
    const std::string e = extent(0, g->lx, 0, g->ly, 0, g->lz);
    return write_vtr(std::string(filename) + ".vtr", e, e, g->lx, g->ly, g->lz, o, len, nscalars, names, fields,
                     static_cast<cudaStream_t>(stream));
}

int mps_write_vtr_piece_dev(const char* dirname, int rank, const int pind[3], const mps_grid* g,
                            const double off[3], int nscalars, const char* const* names,
                            const double* const* fields, void* stream)
{
    if (!dirname || rank < 0 || !pind || !g || g->lx < 1 || g->ly < 1 || g->lz < 1 || !names_ok(nscalars, names) ||
        (nscalars > 0 && !fields) || pind[0] < 1 || pind[1] < 1 || pind[2] < 1)
        return MPS_ERR_BAD_ARG;
    for (int i = 0; i < nscalars; i++)
        if (!fields[i]) return MPS_ERR_BAD_ARG;
    char proc[16];
    std::snprintf(proc, sizeof(proc), "%08d", rank);
    const double o[3] = {off ? off[0] : 0.0, off ? off[1] : 0.0, off ? off[2] : 0.0};
    const double len[3] = {g->llenx, g->lleny, g->llenz};
    const long long lx = g->lx, ly = g->ly, lz = g->lz;
    const std::string e = extent(lx * (pind[0] - 1), lx * pind[0], ly * (pind[1] - 1), ly * pind[1],
                                 lz * (pind[2] - 1), lz * pind[2]);
    return write_vtr(std::string(dirname) + "/file_" + proc + ".vtr", e, e, g->lx, g->ly, g->lz, o, len, nscalars,
                     names, fields, static_cast<cudaStream_t>(stream));
}

int mps_write_pvtr(const char* dirname, const int lxyz[3], const int pxyz[3], int nscalars, const char* const* names)
{
    if (!dirname || !lxyz || !pxyz || !names_ok(nscalars, names)) return MPS_ERR_BAD_ARG;
    for (int a = 0; a < 3; a++)
        if (lxyz[a] < 1 || pxyz[a] < 1) return MPS_ERR_BAD_ARG;
    mkdir(dirname, 0777);  // the reference runs 'mkdir dirname' (:361); an existing folder is fine
    File F(std::string(dirname) + ".pvtr");
    if (!F.ok) return MPS_ERR_BAD_ARG;
    const char nl = '\n';
    const long long lx = lxyz[0], ly = lxyz[1], lz = lxyz[2];
    F.put(std::string("<?xml version=\"1.0\"?>") + nl);
    F.put(std::string("<VTKFile type=\"PRectilinearGrid\" version=\"0.1\" byte_order=\"LittleEndian\">") + nl);
    F.put("<PRectilinearGrid WholeExtent=\"" + extent(0, lx * pxyz[0], 0, ly * pxyz[1], 0, lz * pxyz[2]) +
          "\" GhostLevel=\"0\">" + nl);
    F.put(std::string("<PPointData>  </PPointData>") + nl);
    F.put(std::string("<PCellData> ") + nl);
    for (int i = 0; i < nscalars; i++)
        F.put("<PDataArray type=\"Float64\" Name=\"" + rtrim(names[i]) + "\"/>" + nl);
    F.put(std::string("</PCellData>") + nl);
    F.put(std::string("<PCoordinates>") + nl);
    for (const char* a : {"X", "Y", "Z"}) F.put(std::string("<PDataArray type=\"Float64\" Name=\"") + a + "\"/>" + nl);
    F.put(std::string("</PCoordinates>") + nl);
    // pieces in rank order; rank r+1 -> (pind_x, pind_y, pind_z) as
    // find3dindex (x fastest, globalvars.f90:73-97)
    const int np = pxyz[0] * pxyz[1] * pxyz[2];
    for (int r = 0; r < np; r++) {
        const int px = r % pxyz[0] + 1, py = (r / pxyz[0]) % pxyz[1] + 1, pz = r / (pxyz[0] * pxyz[1]) + 1;
        char proc[16];
        std::snprintf(proc, sizeof(proc), "%08d", r);
        F.put("<Piece Extent=\"" + extent(lx * (px - 1), lx * px, ly * (py - 1), ly * py, lz * (pz - 1), lz * pz) +
              "\" Source=\"" + std::string(dirname) + "/file_" + proc + ".vtr\"/>" + nl);
    }
    F.put(std::string("</PRectilinearGrid>") + nl);
    F.put(std::string("</VTKFile>") + nl);
    return F.ok ? MPS_OK : MPS_ERR_BAD_ARG;
}

}  // extern "C"
