// output.cpp — ParaView output in the reference's layout (io_vtk.c).
//
// One <base>_<ts>.pvtu index (writepvtu, io_vtk.c:39-90) naming one piece
// per subblock, <base>_<sbid>/<ts>.vtu (writevtu, io_vtk.c:203-463): the
// subblock's cells as hexahedral cells (VTK type 11) over the
// (dimx+1)(dimy+1)(dimz+1) grid points at the cell centres' coordinates
// (scoord2realcoord, functions.c:122-139), with the cell arrays Temperature
// (Float64) and Grain (Int32); cells and points run x-major (x outer, z
// inner) as in the reference.  The encoding is the reference's plain-text
// one (its USE_COMPRESSION 0 build): the zlib block encoding is not
// reproduced.
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "mms_internal.h"

using namespace mms;

namespace {

double real_coord(const mms_params &p, int axis, long long c)
{
    return p.origin_offset[axis] + ((double)c + 0.5) * p.cellSize;
}

bool write_pvtu(const mms_params &p, const std::string &base, long long ts)
{
    const std::string fn = base + "_" + std::to_string(ts) + ".pvtu";
    FILE *fp = std::fopen(fn.c_str(), "w");
    if (!fp) return false;
    std::fprintf(fp, "<?xml version=\"1.0\"?>\n");
    std::fprintf(fp, "<VTKFile type=\"PUnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
    std::fprintf(fp, "  <PUnstructuredGrid GhostLevel=\"0\">\n");
    std::fprintf(fp, "    <PCellData>\n");
    std::fprintf(fp, "      <PDataArray type=\"Float64\" Name=\"Temperature\"/>\n");
    std::fprintf(fp, "      <PDataArray type=\"Int32\" Name=\"Grain\"/>\n");
    std::fprintf(fp, "    </PCellData>\n");
    std::fprintf(fp, "    <PPoints>\n");
    std::fprintf(fp, "      <PDataArray type=\"Float32\" NumberOfComponents=\"3\"/>\n");
    std::fprintf(fp, "    </PPoints>\n");
    const int nsub = p.gnsbx * p.gnsby * p.gnsbz;
    for (int s = 0; s < nsub; s++)
        std::fprintf(fp, "    <Piece Source=\"%s_%04d/%lld.vtu\"/>\n", base.c_str(), s, ts);
    std::fprintf(fp, "  </PUnstructuredGrid>\n");
    std::fprintf(fp, "</VTKFile>\n");
    return std::fclose(fp) == 0;
}

// subblock s of the global halo'd arrays (reference layout)
bool write_vtu(const mms_params &p, const std::string &base, long long ts, int s, const double *T, const int *gr)
{
    const int dimx = p.gsdimx, dimy = p.gsdimy, dimz = p.gsdimz;
    const int sx = s % p.gnsbx, sy = (s / p.gnsbx) % p.gnsby, sz = s / (p.gnsbx * p.gnsby);
    const long long gx = (long long)p.gnsbx * dimx, gy = (long long)p.gnsby * dimy;
    const long long rsy = gx + 2, rsz = rsy * (gy + 2);
    char dir[512];
    std::snprintf(dir, sizeof dir, "%s_%04d", base.c_str(), s);
    if (mkdir(dir, 0755) != 0 && errno != EEXIST) return false;
    const std::string fn = std::string(dir) + "/" + std::to_string(ts) + ".vtu";
    FILE *fp = std::fopen(fn.c_str(), "w");
    if (!fp) return false;
    auto gidx = [&](int i, int j, int k) {
        return (long long)(sz * dimz + k) * rsz + (long long)(sy * dimy + j) * rsy + (sx * dimx + i);
    };
    const long long ncells = (long long)dimx * dimy * dimz;
    const long long npoints = (long long)(dimx + 1) * (dimy + 1) * (dimz + 1);
    std::fprintf(fp, "<?xml version=\"1.0\"?>\n");
    std::fprintf(fp, "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
    std::fprintf(fp, "  <UnstructuredGrid>\n");
    std::fprintf(fp, "      <Piece NumberOfPoints=\"%lld\" NumberOfCells=\"%lld\" >\n", npoints, ncells);
    std::fprintf(fp, "        <CellData>\n");
    std::fprintf(fp, "        <DataArray type=\"Float64\" Name=\"Temperature\" format=\"ascii\">\n");
    for (int i = 1; i <= dimx; i++)
        for (int j = 1; j <= dimy; j++)
            for (int k = 1; k <= dimz; k++) std::fprintf(fp, "%lf\n", T[gidx(i, j, k)]);
    std::fprintf(fp, "\n        </DataArray>\n");
    std::fprintf(fp, "        <DataArray type=\"Int32\" Name=\"Grain\" format=\"ascii\">\n");
    for (int i = 1; i <= dimx; i++)
        for (int j = 1; j <= dimy; j++)
            for (int k = 1; k <= dimz; k++) std::fprintf(fp, "%d\n", gr[gidx(i, j, k)]);
    std::fprintf(fp, "\n        </DataArray>\n");
    std::fprintf(fp, "      </CellData>\n");
    std::fprintf(fp, "      <Points>\n");
    std::fprintf(fp, "        <DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    for (int i = 0; i <= dimx; i++)
        for (int j = 0; j <= dimy; j++)
            for (int k = 0; k <= dimz; k++)
                std::fprintf(fp, "%g %g %g\n", (float)real_coord(p, 0, (long long)sx * dimx + i),
                             (float)real_coord(p, 1, (long long)sy * dimy + j),
                             (float)real_coord(p, 2, (long long)sz * dimz + k));
    std::fprintf(fp, "        </DataArray>\n");
    std::fprintf(fp, "      </Points>\n");
    std::fprintf(fp, "      <Cells>\n");
    std::fprintf(fp, "        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n");
    const long long row = dimz + 1, plane = (long long)(dimy + 1) * (dimz + 1);
    for (int i = 0; i < dimx; i++)
        for (int j = 0; j < dimy; j++)
            for (int k = 0; k < dimz; k++) {
                const long long c0 = i * plane + j * row + k;
                std::fprintf(fp, "%lld %lld %lld %lld %lld %lld %lld %lld\n", c0, c0 + 1, c0 + row, c0 + row + 1,
                             c0 + plane, c0 + plane + 1, c0 + plane + row, c0 + plane + row + 1);
            }
    std::fprintf(fp, "        </DataArray>\n");
    std::fprintf(fp, "        <DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n");
    for (long long n = 1; n <= ncells; n++) std::fprintf(fp, "%lld ", n * 8);
    std::fprintf(fp, "\n        </DataArray>\n");
    std::fprintf(fp, "        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n");
    for (long long n = 1; n <= ncells; n++) std::fprintf(fp, "%d ", 11);
    std::fprintf(fp, "\n        </DataArray>\n");
    std::fprintf(fp, "      </Cells>\n");
    std::fprintf(fp, "    </Piece>\n");
    std::fprintf(fp, "  </UnstructuredGrid>\n");
    std::fprintf(fp, "</VTKFile>\n");
    return std::fclose(fp) == 0;
}

}  // namespace

extern "C" mms_status mms_write_vtk_arrays(const mms_params *p, const char *basename, int64_t timestep,
                                           const double *temperature, const int32_t *gr)
{
    if (!p || !basename || !temperature || !gr) return MMS_ERR_ARG;
    const std::string base(basename);
    if (!write_pvtu(*p, base, timestep)) return MMS_ERR_IO;
    const int nsub = p->gnsbx * p->gnsby * p->gnsbz;
    for (int s = 0; s < nsub; s++)
        if (!write_vtu(*p, base, timestep, s, temperature, gr)) return MMS_ERR_IO;
    return MMS_OK;
}

extern "C" mms_status mms_write_vtk(mms_ctx *ctx, const char *basename)
{
    if (!ctx) return MMS_ERR_ARG;
    const mms_params &p = ctx_params(ctx);
    const size_t n = mms_num_cells(ctx);
    std::vector<double> T(n);
    std::vector<int32_t> gr(n);
    mms_status st;
    if ((st = mms_download(ctx, MMS_FIELD_TEMPERATURE, T.data())) || (st = mms_download(ctx, MMS_FIELD_GR, gr.data())))
        return st;
    uint64_t ts = 0;
    if ((st = mms_get_timestep(ctx, &ts))) return st;
    return mms_write_vtk_arrays(&p, basename ? basename : p.basefilename, (int64_t)ts, T.data(), gr.data());
}
