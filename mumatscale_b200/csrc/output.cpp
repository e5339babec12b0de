// output.cpp — ParaView output in the reference's layout (io_vtk.c).
//
// One <base>_<ts>.pvtu index (writepvtu, io_vtk.c:39-90) naming one piece
// per subblock, <base>_<sbid>/<ts>.vtu (writevtu, io_vtk.c:203-463): the
// subblock's cells as hexahedral cells (VTK type 11) over the
// (dimx+1)(dimy+1)(dimz+1) grid points at the cell centres' coordinates
// (scoord2realcoord, functions.c:122-139), with the cell arrays Temperature
// (Float64) and Grain (Int32); cells and points run x-major (x outer, z
// inner) as in the reference.
//
// Encoding: the reference's default build (USE_COMPRESSION 1,
// io_vtk.c:20-22; its plain-text branch does not compile), VTK's "binary"
// format with vtkZLibDataCompressor.  Every data array is a list of blocks
// (one per x plane of the subblock, or one block for offsets and types),
// each compressed on its own with zlib's compress(); the array is written as
// the base64 text of its header, uint32 {number of blocks, block size, 0,
// compressed size of each block}, followed by the base64 text of the
// concatenated compressed blocks (vtkCompress.c:86-129).  With the same zlib
// the files are byte-identical to the reference's.
#include <zlib.h>

#include <cerrno>
#include <cstdint>
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

// Base64 (RFC 4648 alphabet, '=' padding) of len bytes.
void put_base64(FILE *fp, const unsigned char *d, size_t len)
{
    static const char tab[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
    std::string out;
    out.reserve((len + 2) / 3 * 4);
    for (size_t i = 0; i < len; i += 3) {
        const size_t n = len - i < 3 ? len - i : 3;
        const unsigned v = (unsigned)d[i] << 16 | (n > 1 ? (unsigned)d[i + 1] << 8 : 0u) | (n > 2 ? d[i + 2] : 0u);
        out += tab[(v >> 18) & 63];
        out += tab[(v >> 12) & 63];
        out += n > 1 ? tab[(v >> 6) & 63] : '=';
        out += n > 2 ? tab[v & 63] : '=';
    }
    std::fwrite(out.data(), 1, out.size(), fp);
}

// One data array in VTK's zlib block encoding.
struct ZBlocks {
    std::vector<uint32_t> hdr{0, 0, 0};  // blocks, block size, last-block size (0: full)
    std::vector<unsigned char> data;
    std::vector<unsigned char> tmp;
    bool ok = true;
    void add(const void *p, uint32_t len)
    {
        if (hdr[0] == 0) hdr[1] = len;
        else if (len != hdr[1]) ok = false;
        hdr[0]++;
        uLongf n = compressBound(len);
        tmp.resize(n);
        if (compress(tmp.data(), &n, (const Bytef *)p, len) != Z_OK) ok = false;
        hdr.push_back((uint32_t)n);
        data.insert(data.end(), tmp.begin(), tmp.begin() + n);
    }
    bool write(FILE *fp) const
    {
        put_base64(fp, (const unsigned char *)hdr.data(), hdr.size() * sizeof(uint32_t));
        put_base64(fp, data.data(), data.size());
        return ok;
    }
};

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
    std::fprintf(fp, "      <PDataArray type=\"Float64\" NumberOfComponents=\"3\"/>\n");
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
    bool ok = true;
    std::fprintf(fp, "<?xml version=\"1.0\"?>\n");
    std::fprintf(fp, "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\" "
                     "compressor=\"vtkZLibDataCompressor\">\n");
    std::fprintf(fp, "  <UnstructuredGrid>\n");
    std::fprintf(fp, "      <Piece NumberOfPoints=\"%lld\" NumberOfCells=\"%lld\" >\n", npoints, ncells);
    std::fprintf(fp, "        <CellData>\n");
    {
        // writeDataArrayFloat / writeDataArrayInt32: one block per x plane
        ZBlocks bt, bg;
        std::vector<double> tv((size_t)dimy * dimz);
        std::vector<int32_t> gv((size_t)dimy * dimz);
        for (int i = 1; i <= dimx; i++) {
            size_t n = 0;
            for (int j = 1; j <= dimy; j++)
                for (int k = 1; k <= dimz; k++, n++) {
                    tv[n] = T[gidx(i, j, k)];
                    gv[n] = gr[gidx(i, j, k)];
                }
            bt.add(tv.data(), (uint32_t)(tv.size() * sizeof(double)));
            bg.add(gv.data(), (uint32_t)(gv.size() * sizeof(int32_t)));
        }
        std::fprintf(fp, "        <DataArray type=\"Float64\" Name=\"Temperature\" format=\"binary\">\n");
        ok &= bt.write(fp);
        std::fprintf(fp, "\n        </DataArray>\n");
        std::fprintf(fp, "        <DataArray type=\"Int32\" Name=\"Grain\" format=\"binary\">\n");
        ok &= bg.write(fp);
        std::fprintf(fp, "\n        </DataArray>\n");
    }
    std::fprintf(fp, "      </CellData>\n");
    std::fprintf(fp, "      <Points>\n");
    std::fprintf(fp, "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"binary\">\n");
    {
        ZBlocks b;
        std::vector<double> v((size_t)3 * (dimy + 1) * (dimz + 1));
        for (int i = 0; i <= dimx; i++) {
            size_t n = 0;
            for (int j = 0; j <= dimy; j++)
                for (int k = 0; k <= dimz; k++) {
                    v[n++] = real_coord(p, 0, (long long)sx * dimx + i);
                    v[n++] = real_coord(p, 1, (long long)sy * dimy + j);
                    v[n++] = real_coord(p, 2, (long long)sz * dimz + k);
                }
            b.add(v.data(), (uint32_t)(v.size() * sizeof(double)));
        }
        ok &= b.write(fp);
    }
    std::fprintf(fp, "        </DataArray>\n");
    std::fprintf(fp, "      </Points>\n");
    std::fprintf(fp, "      <Cells>\n");
    std::fprintf(fp, "        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"binary\">\n");
    {
        ZBlocks b;
        std::vector<int32_t> v((size_t)dimy * dimz * 8);
        const int row = dimz + 1, plane = (dimy + 1) * (dimz + 1);
        for (int i = 0; i < dimx; i++) {
            size_t n = 0;
            for (int j = 0; j < dimy; j++)
                for (int k = 0; k < dimz; k++) {
                    const int c0 = i * plane + j * row + k;
                    const int32_t q[8] = {c0, c0 + 1, c0 + row, c0 + row + 1,
                                          c0 + plane, c0 + plane + 1, c0 + plane + row, c0 + plane + row + 1};
                    for (int e = 0; e < 8; e++) v[n++] = q[e];
                }
            b.add(v.data(), (uint32_t)(v.size() * sizeof(int32_t)));
        }
        ok &= b.write(fp);
    }
    std::fprintf(fp, "        </DataArray>\n");
    std::fprintf(fp, "        <DataArray type=\"Int32\" Name=\"offsets\" format=\"binary\">\n");
    {
        ZBlocks b;
        std::vector<int32_t> v((size_t)ncells);
        for (long long n = 1; n <= ncells; n++) v[n - 1] = (int32_t)(n * 8);
        b.add(v.data(), (uint32_t)(v.size() * sizeof(int32_t)));
        ok &= b.write(fp);
    }
    std::fprintf(fp, "        </DataArray>\n");
    std::fprintf(fp, "        <DataArray type=\"UInt8\" Name=\"types\" format=\"binary\">\n");
    {
        ZBlocks b;
        std::vector<unsigned char> v((size_t)ncells, 11);  // VTK_VOXEL
        b.add(v.data(), (uint32_t)v.size());
        ok &= b.write(fp);
    }
    std::fprintf(fp, "        </DataArray>\n");
    std::fprintf(fp, "       </Cells>\n");
    std::fprintf(fp, "    </Piece>\n");
    std::fprintf(fp, "  </UnstructuredGrid>\n");
    std::fprintf(fp, "</VTKFile>\n");
    return (std::fclose(fp) == 0) && ok;
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

// ------------------------------------------------------------------- XDMF
// The reference's XDMF output (io_xdmf.c): a time-series index
// <base>_ts.xmf (writeXDMFTimeSeries, io_xdmf.c:483-497, grids as
// writeXDMFGrids, io_xdmf.c:141-305, global items as writeGlobalData,
// io_xdmf.c:378-404), per-rank heavy data <base>_r<rank>/<ts>.raw
// (xdmf_writeSubblocks, io_xdmf.c:561-673: Temperature, CE, Grain,
// FracSolid of the subblock's interior, float32 / int32, z slowest) and the
// global grain data <base>_gbl.raw (writeGlobalHeavyData, io_xdmf.c:408-468:
// GrainRenumber as uint64 when RandomizeGrains, then GrainAngleX/Y/Z as
// float32).  libhdf5 is absent, so each dataset is a little-endian block of
// a raw file that the index addresses with Format="Binary" and a Seek
// offset; the index states each block's true number type (the reference's
// index says Precision 8 for datasets it writes as float32).
namespace {

std::string local_name(const std::string &base)
{
    const size_t k = base.rfind('/');
    return k == std::string::npos ? base : base.substr(k + 1);
}

std::string rank_file(const std::string &base, int rank, long long ts)
{
    char buf[64];
    std::snprintf(buf, sizeof buf, "_r%d/%05lld.raw", rank, ts);
    return base + buf;
}

bool write_all(FILE *fp, const void *p, size_t n) { return n == 0 || std::fwrite(p, 1, n, fp) == n; }

// one subblock's interior of the global halo'd arrays, as the four blocks
bool write_rank_raw(const mms_params &p, const std::string &base, long long ts, int s, const double *T,
                    const double *ce, const int32_t *gr, const double *fs)
{
    const int dimx = p.gsdimx, dimy = p.gsdimy, dimz = p.gsdimz;
    const int sx = s % p.gnsbx, sy = (s / p.gnsbx) % p.gnsby, sz = s / (p.gnsbx * p.gnsby);
    const long long gx = (long long)p.gnsbx * dimx, gy = (long long)p.gnsby * dimy;
    const long long rsy = gx + 2, rsz = rsy * (gy + 2);
    char dir[600];
    std::snprintf(dir, sizeof dir, "%s_r%d", base.c_str(), s);
    if (mkdir(dir, 0755) != 0 && errno != EEXIST) return false;
    FILE *fp = std::fopen(rank_file(base, s, ts).c_str(), "wb");
    if (!fp) return false;
    const size_t n = (size_t)dimx * dimy * dimz;
    std::vector<float> f(n);
    std::vector<int32_t> g(n);
    auto each = [&](auto fn) {
        size_t q = 0;
        for (int k = 1; k <= dimz; k++)
            for (int j = 1; j <= dimy; j++)
                for (int i = 1; i <= dimx; i++, q++)
                    fn(q, (long long)(sz * dimz + k) * rsz + (long long)(sy * dimy + j) * rsy + (sx * dimx + i));
    };
    bool ok = true;
    each([&](size_t q, long long c) { f[q] = (float)T[c]; });
    ok = ok && write_all(fp, f.data(), n * sizeof(float));
    each([&](size_t q, long long c) { f[q] = (float)ce[c]; });
    ok = ok && write_all(fp, f.data(), n * sizeof(float));
    each([&](size_t q, long long c) { g[q] = gr[c]; });
    ok = ok && write_all(fp, g.data(), n * sizeof(int32_t));
    each([&](size_t q, long long c) { f[q] = (float)fs[c]; });
    ok = ok && write_all(fp, f.data(), n * sizeof(float));
    return (std::fclose(fp) == 0) && ok;
}

bool write_global_raw(const std::string &base, int ng, const double *rotang, const uint64_t *renumber)
{
    FILE *fp = std::fopen((base + "_gbl.raw").c_str(), "wb");
    if (!fp) return false;
    bool ok = true;
    if (renumber) ok = write_all(fp, renumber, (size_t)ng * sizeof(uint64_t));
    std::vector<float> a((size_t)ng);
    for (int d = 0; d < 3 && ok; d++) {
        for (int i = 0; i < ng; i++) a[i] = (float)rotang[3 * (size_t)i + d];
        ok = write_all(fp, a.data(), a.size() * sizeof(float));
    }
    return (std::fclose(fp) == 0) && ok;
}

void xmf_block(FILE *fp, const char *ind, const char *type, int prec, long long seek, const mms_params &p,
               const std::string &file)
{
    std::fprintf(fp,
                 "%s<DataItem Format=\"Binary\" Endian=\"Little\" Seek=\"%lld\" NumberType=\"%s\" Precision=\"%d\" "
                 "Dimensions=\"%d %d %d\">\n",
                 ind, seek, type, prec, p.gsdimz, p.gsdimy, p.gsdimx);
    std::fprintf(fp, "%s\t%s\n", ind, file.c_str());
    std::fprintf(fp, "%s</DataItem>\n", ind);
}

void xmf_grids(FILE *fp, const mms_params &p, const std::string &lbase, long long ts, bool renumber)
{
    const char *ind = "\t\t\t";
    const double t = (double)ts * p.ts_delt;
    const long long n = (long long)p.gsdimx * p.gsdimy * p.gsdimz;
    std::fprintf(fp, "%s<Grid Name=\"Full Volume at time %g\" GridType=\"Collection\" CollectionType=\"Spatial\">\n",
                 ind, t);
    std::fprintf(fp, "%s\t<Time Value=\"%g\" />\n", ind, t);
    const int nsub = p.gnsbx * p.gnsby * p.gnsbz;
    for (int s = 0; s < nsub; s++) {
        const int cx = s % p.gnsbx, cy = (s / p.gnsbx) % p.gnsby, cz = s / (p.gnsbx * p.gnsby);
        const std::string file = rank_file(lbase, s, ts);
        std::fprintf(fp, "%s\t<Grid Name=\"SubBlock %dx%dx%d (%d)\" GridType=\"Uniform\">\n", ind, cx, cy, cz, s);
        std::fprintf(fp, "%s\t\t<Topology TopologyType=\"3DCoRectMesh\" Dimensions=\"%u %u %u\" />\n", ind,
                     p.gsdimz + 1, p.gsdimy + 1, p.gsdimx + 1);
        std::fprintf(fp, "%s\t\t<Geometry GeometryType=\"ORIGIN_DXDYDZ\">\n", ind);
        std::fprintf(fp, "%s\t\t\t<DataItem Format=\"XML\" Dimensions=\"3\">\n", ind);
        // getSBRealBounds (functions.c:153-173): the subblock's first cell
        // centre less half a cell, printed z y x
        const double rx = real_coord(p, 0, (long long)cx * p.gsdimx) - p.cellSize / 2.0;
        const double ry = real_coord(p, 1, (long long)cy * p.gsdimy) - p.cellSize / 2.0;
        const double rz = real_coord(p, 2, (long long)cz * p.gsdimz) - p.cellSize / 2.0;
        std::fprintf(fp, "%s\t\t\t\t%e %e %e\n", ind, rz, ry, rx);
        std::fprintf(fp, "%s\t\t\t</DataItem>\n", ind);
        std::fprintf(fp, "%s\t\t\t<DataItem Format=\"XML\" Dimensions=\"3\">\n", ind);
        std::fprintf(fp, "%s\t\t\t\t%e %e %e\n", ind, p.cellSize, p.cellSize, p.cellSize);
        std::fprintf(fp, "%s\t\t\t</DataItem>\n", ind);
        std::fprintf(fp, "%s\t\t</Geometry>\n", ind);
        const std::string a = std::string(ind) + "\t\t\t";
        std::fprintf(fp, "%s\t\t<Attribute Name=\"Temperature\" Center=\"Cell\">\n", ind);
        xmf_block(fp, a.c_str(), "Float", 4, 0, p, file);
        std::fprintf(fp, "%s\t\t</Attribute>\n", ind);
        std::fprintf(fp, "%s\t\t<Attribute Name=\"Solute Composition\" Center=\"Cell\">\n", ind);
        xmf_block(fp, a.c_str(), "Float", 4, 4 * n, p, file);
        std::fprintf(fp, "%s\t\t</Attribute>\n", ind);
        std::fprintf(fp, "%s\t\t<Attribute Name=\"Grain\" Center=\"Cell\">\n", ind);
        const std::string a2 = a + "\t";
        if (renumber) {
            std::fprintf(fp,
                         "%s<DataItem ItemType=\"Function\" NumberType=\"UInt\" Dimensions=\"%u %u %u\" "
                         "Function=\"$0[$1]\">\n",
                         a.c_str(), p.gsdimz, p.gsdimy, p.gsdimx);
            std::fprintf(fp, "%s<DataItem Reference=\"XML\" Dimensions=\"%u %u %u\">\n", a2.c_str(), p.gsdimz, p.gsdimy,
                         p.gsdimx);
            std::fprintf(fp, "%s\t/Xdmf/Domain/DataItem[@Name=\"Grain Renumber\"]\n", a2.c_str());
            std::fprintf(fp, "%s</DataItem>\n", a2.c_str());
            xmf_block(fp, a2.c_str(), "Int", 4, 8 * n, p, file);
            std::fprintf(fp, "%s</DataItem>\n", a.c_str());
        } else {
            xmf_block(fp, a.c_str(), "Int", 4, 8 * n, p, file);
        }
        std::fprintf(fp, "%s\t\t</Attribute>\n", ind);
        std::fprintf(fp, "%s\t\t<Attribute Name=\"Grain Angle\" Center=\"Cell\" AttributeType=\"Vector\">\n", ind);
        std::fprintf(fp,
                     "%s<DataItem ItemType=\"Function\" NumberType=\"Float\" Dimensions=\"%u %u %u 3\" "
                     "Function=\"$1[$0], $2[$0], $3[$0]\">\n",
                     a.c_str(), p.gsdimz, p.gsdimy, p.gsdimx);
        xmf_block(fp, a2.c_str(), "Int", 4, 8 * n, p, file);
        for (char d : {'X', 'Y', 'Z'}) {
            std::fprintf(fp, "%s<DataItem Reference=\"XML\" Dimensions=\"%u %u %u\">\n", a2.c_str(), p.gsdimz, p.gsdimy,
                         p.gsdimx);
            std::fprintf(fp, "%s\t/Xdmf/Domain/DataItem[@Name=\"Grain Angle %c\"]\n", a2.c_str(), d);
            std::fprintf(fp, "%s</DataItem>\n", a2.c_str());
        }
        std::fprintf(fp, "%s</DataItem>\n", a.c_str());
        std::fprintf(fp, "%s\t\t</Attribute>\n", ind);
        std::fprintf(fp, "%s\t\t<Attribute Name=\"Fraction Solid\" Center=\"Cell\">\n", ind);
        xmf_block(fp, a.c_str(), "Float", 4, 12 * n, p, file);
        std::fprintf(fp, "%s\t\t</Attribute>\n", ind);
        std::fprintf(fp, "%s\t</Grid>\n", ind);
    }
    std::fprintf(fp, "%s</Grid>\n", ind);
}

bool write_xmf(const mms_params &p, const std::string &base, const int64_t *series, int nseries, int ng,
               bool renumber)
{
    FILE *fp = std::fopen((base + "_ts.xmf").c_str(), "w");
    if (!fp) return false;
    const std::string lbase = local_name(base);
    std::fprintf(fp, "<?xml version=\"1.0\" ?>\n");
    std::fprintf(fp, "<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n");
    std::fprintf(fp, "<Xdmf xmlns:xi=\"http://www.w3.org/2001/XInclude\" Version=\"2.0\">\n");
    std::fprintf(fp, "\t<Domain>\n");
    std::fprintf(fp, "\t\t<Information Name=\"Description\">\n");
    std::fprintf(fp, "\t\t\tSimulation time series data\n");
    std::fprintf(fp, "\t\t</Information>\n");
    std::fprintf(fp, "\t\t<Grid Name=\"Time Series\" GridType=\"Collection\" CollectionType=\"Temporal\">\n");
    for (int i = 0; i < nseries; i++) xmf_grids(fp, p, lbase, (long long)series[i], renumber);
    std::fprintf(fp, "\t\t</Grid>\n");
    const std::string gfile = lbase + "_gbl.raw";
    long long off = 0;
    if (renumber) {
        std::fprintf(fp,
                     "\t\t<DataItem Name=\"Grain Renumber\" Format=\"Binary\" Endian=\"Little\" Seek=\"0\" "
                     "Dimensions=\"%d\" NumberType=\"UInt\" Precision=\"8\">\n",
                     ng);
        std::fprintf(fp, "\t\t\t%s\n\t\t</DataItem>\n", gfile.c_str());
        off = 8LL * ng;
    }
    for (char d : {'X', 'Y', 'Z'}) {
        std::fprintf(fp,
                     "\t\t<DataItem Name=\"Grain Angle %c\" Format=\"Binary\" Endian=\"Little\" Seek=\"%lld\" "
                     "Dimensions=\"%d\" NumberType=\"Float\" Precision=\"4\">\n",
                     d, off, ng);
        std::fprintf(fp, "\t\t\t%s\n\t\t</DataItem>\n", gfile.c_str());
        off += 4LL * ng;
    }
    std::fprintf(fp, "\t</Domain>\n");
    std::fprintf(fp, "</Xdmf>\n");
    return std::fclose(fp) == 0;
}

}  // namespace

extern "C" mms_status mms_write_xdmf_arrays(const mms_params *p, const char *basename, const int64_t *series,
                                            int nseries, const double *temperature, const double *ce,
                                            const int32_t *gr, const double *fs, int num_grains,
                                            const double *rotang, const uint64_t *renumber)
{
    if (!p || !basename || !series || nseries < 1 || !temperature || !ce || !gr || !fs || num_grains < 1 ||
        !rotang)
        return MMS_ERR_ARG;
    const std::string base(basename);
    const long long ts = (long long)series[nseries - 1];
    const int nsub = p->gnsbx * p->gnsby * p->gnsbz;
    for (int s = 0; s < nsub; s++)
        if (!write_rank_raw(*p, base, ts, s, temperature, ce, gr, fs)) return MMS_ERR_IO;
    if (!write_global_raw(base, num_grains, rotang, renumber)) return MMS_ERR_IO;
    if (!write_xmf(*p, base, series, nseries, num_grains, renumber != nullptr)) return MMS_ERR_IO;
    return MMS_OK;
}
