// dare_vtk.cu -- field output in the VTK XML parallel structured-grid format
// (host code; no kernels).
//
// Writes what the reference's io::VTKWriter<Cartesian<Dim>> writes for one
// grid on one rank (IO/VTKWriter.inl:34-86, Grid/Cartesian/VTKOptions_Cartesian.h:146-323,
// IO/VTKPXMLStructuredGridWriter.cpp:32-45, IO/VTKWriter.cpp:29-47):
//   <base>/<grid>_<step>.pvts                 PStructuredGrid, GhostLevel = num_ghost,
//                                             one Piece (Source, then Extent)
//   <base>/<grid>_<step>/<grid>_<step>_0.vts  StructuredGrid piece
// The grid is the local grid INCLUDING its ghost layers: (n + 2 g) cells per
// active dimension, extent 0 .. n + 2 g, node coordinates x_i = dx i - g dx
// (Float32, as vtkPoints stores them by default), 1-D grids written as a
// pseudo-2-D grid one cell high (dy = dx), inactive dimensions with one node
// layer.  Cell arrays are Float64, ordered x fastest (VTK's order; the grid's
// own numbering has the last dimension fastest), one tuple per ghosted cell;
// a time >= 0 is stored as the field array "TimeValue".  Arrays are written
// inline in VTK's "binary" encoding (base64 of a UInt64 byte count, then
// base64 of the little-endian data), uncompressed; VTK and ParaView read it.
#include <cuda_runtime.h>
#include <errno.h>
#include <sys/stat.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "dare_internal.cuh"

namespace {

std::string base64(const uint8_t* p, size_t n) {
    static const char* tab = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
    std::string out;
    out.reserve((n + 2) / 3 * 4);
    size_t i = 0;
    for (; i + 2 < n; i += 3) {
        const uint32_t v = (uint32_t)p[i] << 16 | (uint32_t)p[i + 1] << 8 | p[i + 2];
        out += tab[v >> 18];
        out += tab[(v >> 12) & 63];
        out += tab[(v >> 6) & 63];
        out += tab[v & 63];
    }
    if (i < n) {
        const uint32_t v = (uint32_t)p[i] << 16 | (i + 1 < n ? (uint32_t)p[i + 1] << 8 : 0u);
        out += tab[v >> 18];
        out += tab[(v >> 12) & 63];
        out += i + 1 < n ? tab[(v >> 6) & 63] : '=';
        out += '=';
    }
    return out;
}

// VTK inline binary: the UInt64 byte count and the data, each base64-encoded
std::string vtk_binary(const void* data, size_t bytes) {
    const uint64_t header = bytes;
    return base64(reinterpret_cast<const uint8_t*>(&header), sizeof(header)) +
           base64(reinterpret_cast<const uint8_t*>(data), bytes);
}

std::string fmt_double(double v) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.17g", v);
    return buf;
}

template <typename T>
void range_of(const std::vector<T>& v, int ncomp, double* lo, double* hi) {
    // VTK's RangeMin/RangeMax: of the values (1 component) or of the tuple
    // magnitudes (several components)
    *lo = std::numeric_limits<double>::infinity();
    *hi = -std::numeric_limits<double>::infinity();
    for (size_t t = 0; t * ncomp < v.size(); t++) {
        double m;
        if (ncomp == 1) {
            m = (double)v[t];
        } else {
            double s = 0.;
            for (int c = 0; c < ncomp; c++) s += (double)v[t * ncomp + c] * (double)v[t * ncomp + c];
            m = std::sqrt(s);
        }
        if (m < *lo) *lo = m;
        if (m > *hi) *hi = m;
    }
}

bool make_dir(const std::string& path) {
    if (path.empty()) return true;
    if (mkdir(path.c_str(), 0775) == 0 || errno == EEXIST) return true;
    return false;
}

struct Geometry {
    int dim = 0, ng = 0;
    int64_t ext[3] = {0, 0, 0};    // extent maxima (cells; 0 for a single node layer)
    double dn[3] = {0., 0., 0.};
    double off[3] = {0., 0., 0.};
};

Geometry make_geometry(int dim, const int64_t n[3], const double dn[3], const double origin[3], int ng) {
    Geometry G;
    G.dim = dim;
    G.ng = ng;
    for (int d = 0; d < dim; d++) {
        G.ext[d] = n[d] + 2 * ng;
        G.dn[d] = dn[d];
        G.off[d] = origin[d] - (double)ng * G.dn[d];   // offset_size - num_ghost * dn (VTKOptions_Cartesian.h:160-162)
    }
    if (dim == 1) {                                 // pseudo 2-D grid for 1-D (VTKOptions_Cartesian.h:172-176)
        G.ext[1] = 1;
        G.dn[1] = G.dn[0];
    }
    return G;
}

std::string extent_str(const Geometry& G) {
    std::ostringstream os;
    os << 0 << ' ' << G.ext[0] << ' ' << 0 << ' ' << G.ext[1] << ' ' << 0 << ' ' << G.ext[2];
    return os.str();
}

int write_vtk(int dim, const int64_t n[3], const double dn[3], const double origin[3], int num_ghost,
              const double* const* data,
              const char* const* names, int count, const char* base_path, const char* grid_name, int step,
              double time) {
    if (!data || !names || count < 1 || !base_path || !grid_name || !grid_name[0]) return DARE_ERR_BAD_ARG;
    for (int f = 0; f < count; f++)
        if (!data[f] || !names[f] || !names[f][0]) return DARE_ERR_BAD_ARG;
    const Geometry G = make_geometry(dim, n, dn, origin, num_ghost);

    // the grid's ghosted numbering: (i gn1 + j) gn2 + k over its active dims
    int64_t gn[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) gn[d] = n[d] + 2 * num_ghost;
    const int64_t ncell = gn[0] * gn[1] * gn[2];

    // node coordinates, x fastest (VTKOptions_Cartesian.h:185-197)
    const int64_t px = G.ext[0] + 1, py = G.ext[1] + 1, pz = G.ext[2] + 1;
    std::vector<float> pts;
    pts.reserve(px * py * pz * 3);
    for (int64_t k = 0; k < pz; k++)
        for (int64_t j = 0; j < py; j++)
            for (int64_t i = 0; i < px; i++) {
                pts.push_back((float)(G.dn[0] * (double)i + G.off[0]));
                pts.push_back((float)(G.dn[1] * (double)j + G.off[1]));
                pts.push_back((float)(G.dn[2] * (double)k + G.off[2]));
            }

    const std::string name = std::string(grid_name) + "_" + std::to_string(step);
    std::string base = base_path;
    if (!base.empty() && base.back() != '/') base += '/';
    if (!make_dir(base_path) || !make_dir(base + name)) return DARE_ERR_BAD_ARG;
    const std::string piece_rel = name + "/" + name + "_0.vts";

    // ---- the piece ----
    {
        std::ofstream os(base + piece_rel, std::ios::binary);
        if (!os) return DARE_ERR_BAD_ARG;
        const std::string ext = extent_str(G);
        os << "<?xml version=\"1.0\"?>\n"
           << "<VTKFile type=\"StructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n"
           << "  <StructuredGrid WholeExtent=\"" << ext << "\">\n";
        if (time >= 0.) {                           // VTKWriter.inl:135-144
            os << "    <FieldData>\n"
               << "      <DataArray type=\"Float64\" Name=\"TimeValue\" NumberOfTuples=\"1\" format=\"binary\">\n"
               << "        " << vtk_binary(&time, sizeof(double)) << "\n"
               << "      </DataArray>\n"
               << "    </FieldData>\n";
        }
        os << "    <Piece Extent=\"" << ext << "\">\n"
           << "      <PointData>\n      </PointData>\n"
           << "      <CellData>\n";
        std::vector<double> v(ncell);
        for (int f = 0; f < count; f++) {
            // vtk id = i + j cx + k cx cy (VTKOptions_Cartesian.h:67-111)
            int64_t t = 0;
            for (int64_t k = 0; k < gn[2]; k++)
                for (int64_t j = 0; j < gn[1]; j++)
                    for (int64_t i = 0; i < gn[0]; i++) v[t++] = data[f][(i * gn[1] + j) * gn[2] + k];
            double lo, hi;
            range_of(v, 1, &lo, &hi);
            os << "        <DataArray type=\"Float64\" Name=\"" << names[f] << "\" format=\"binary\" RangeMin=\""
               << fmt_double(lo) << "\" RangeMax=\"" << fmt_double(hi) << "\">\n"
               << "          " << vtk_binary(v.data(), v.size() * sizeof(double)) << "\n"
               << "        </DataArray>\n";
        }
        double lo, hi;
        range_of(pts, 3, &lo, &hi);
        os << "      </CellData>\n"
           << "      <Points>\n"
           << "        <DataArray type=\"Float32\" Name=\"Points\" NumberOfComponents=\"3\" format=\"binary\" RangeMin=\""
           << fmt_double(lo) << "\" RangeMax=\"" << fmt_double(hi) << "\">\n"
           << "          " << vtk_binary(pts.data(), pts.size() * sizeof(float)) << "\n"
           << "        </DataArray>\n"
           << "      </Points>\n"
           << "    </Piece>\n"
           << "  </StructuredGrid>\n"
           << "</VTKFile>\n";
        if (!os) return DARE_ERR_BAD_ARG;
    }
    // ---- the parallel root file (one piece on one rank; no halo correction:
    // a single rank owns every boundary, VTKOptions_Cartesian.h:232-246) ----
    {
        std::ofstream os(base + name + ".pvts", std::ios::binary);
        if (!os) return DARE_ERR_BAD_ARG;
        const std::string ext = extent_str(G);
        os << "<?xml version=\"1.0\"?>\n"
           << "<VTKFile type=\"PStructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n"
           << "  <PStructuredGrid WholeExtent=\"" << ext << "\" GhostLevel=\"" << num_ghost << "\">\n"
           << "    <PPointData>\n    </PPointData>\n"
           << "    <PCellData>\n";
        for (int f = 0; f < count; f++) os << "      <PDataArray type=\"Float64\" Name=\"" << names[f] << "\"/>\n";
        os << "    </PCellData>\n"
           << "    <PPoints>\n"
           << "      <PDataArray type=\"Float32\" Name=\"Points\" NumberOfComponents=\"3\"/>\n"
           << "    </PPoints>\n"
           << "    <Piece Source=\"" << piece_rel << "\" Extent=\"" << ext << "\"/>\n"
           << "  </PStructuredGrid>\n"
           << "</VTKFile>\n";
        if (!os) return DARE_ERR_BAD_ARG;
    }
    return DARE_OK;
}

}  // namespace

extern "C" int dare_vtk_write_host(int dim, const int64_t n[3], const double size[3], int num_ghost,
                                   const double* const* data, const char* const* names, int count,
                                   const char* base_path, const char* grid_name, int step, double time) {
    if (dim < 1 || dim > 3 || !n || !size || num_ghost < 0) return DARE_ERR_BAD_ARG;
    int64_t nn[3] = {1, 1, 1};
    double dn[3] = {0., 0., 0.};
    for (int d = 0; d < dim; d++) {
        if (n[d] < 1 || !(size[d] > 0.)) return DARE_ERR_BAD_ARG;
        nn[d] = n[d];
        dn[d] = size[d] / (double)n[d];  // cell width, CartesianMesh.inl:75-77
    }
    const double origin[3] = {0., 0., 0.};
    return write_vtk(dim, nn, dn, origin, num_ghost, data, names, count, base_path, grid_name, step, time);
}

extern "C" int dare_vtk_write(dare_field* const* fields, int level, const char* const* names, int count,
                              const char* base_path, const char* grid_name, int step, double time) {
    if (!fields || count < 1 || !fields[0]) return DARE_ERR_BAD_ARG;
    dare_grid* g = fields[0]->grid;
    for (int f = 0; f < count; f++)
        if (!fields[f] || fields[f]->grid != g || level < 0 || level >= fields[f]->num_levels) return DARE_ERR_BAD_ARG;
    dare_ctx* ctx = g->ctx;
    cudaSetDevice(ctx->device);
    const dare_gpu::GridDev& d = g->dev;
    std::vector<std::vector<double>> host(count, std::vector<double>(d.ncell_ghosted));
    std::vector<const double*> ptr(count);
    for (int f = 0; f < count; f++) {
        DARE_CUDA(ctx, cudaMemcpyAsync(host[f].data(), fields[f]->level[level], d.ncell_ghosted * sizeof(double),
                                       cudaMemcpyDeviceToHost, ctx->stream));
        ptr[f] = host[f].data();
    }
    DARE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    int64_t n[3] = {1, 1, 1};
    double dn[3] = {0., 0., 0.};
    for (int k = 0; k < d.dim; k++) {
        n[k] = d.n[k];
        dn[k] = d.dx[k];
    }
    const int rc = write_vtk(d.dim, n, dn, d.origin, d.ng, ptr.data(), names, count, base_path, grid_name, step, time);
    if (rc) return dare_gpu::set_error(ctx, rc, "dare_vtk_write: cannot write to the output path");
    return DARE_OK;
}
