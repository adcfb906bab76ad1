// Checkpoint/resume files and ParaView output of a DGSEM state (host code).
//
// Checkpoints follow the reference's layout (Simulation.cpp:1084-1116 save,
// :350-384 load):
//   <folder>/Cycle<ti>/checkpoint_cycle_<ti>.<rank, 8 digits>.chk
//       an MFEM GridFunction in text form: the FiniteElementSpace header
//       (L2_T1_<dim>D_P<order>, VDim dim+2, Ordering 0 = byNODES) and one value
//       per line;
//   <folder>/Cycle<ti>/checkpoint_cycle_<ti>.json   {"time": t, "cycle": ti}
// Values and time are written with 17 significant digits, so a save / load
// round trip is exact (the reference's streams keep their default precision:
// 6 digits for the values, 6 decimals for the time).  The loader reads either
// ordering and any precision, and checks the cycle in the meta file as the
// reference does.
//
// ParaView output follows the reference's ParaViewDataCollection setup
// (Simulation.cpp:389-410: high-order output, levels of detail = order):
//   <dir>/<name>/<name>.pvd, <dir>/<name>/Cycle<6 digits>/data.pvtu and
//   proc000000.vtu, unstructured grids of VTK Lagrange quadrilaterals /
//   hexahedra of the mesh order with point fields "Density", "Horizontal V",
//   "Vertical V", "Normal V" (3D), "Pressure" and "Blending Coeff".  The
//   nodal (Gauss-Lobatto) solution is interpolated to the cells' equispaced
//   points; the geometry is affine, so node coordinates interpolate exactly.
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/prandtl_b200.h"

namespace {

thread_local std::string g_io_error;

prandtl_status io_fail(prandtl_status st, const std::string &msg) {
    g_io_error = msg;
    return st;
}

bool make_dirs(const std::string &path) {
    std::string cur;
    for (size_t i = 0; i <= path.size(); ++i) {
        if (i == path.size() || path[i] == '/') {
            if (!cur.empty() && cur != "." && cur != "..") {
                if (mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) return false;
            }
        }
        if (i < path.size()) cur += path[i];
    }
    return true;
}

std::string cycle_dir(const char *folder, int cycle) { return std::string(folder) + "/Cycle" + std::to_string(cycle); }

std::string chk_name(const char *folder, int cycle, int rank) {
    char r[16];
    std::snprintf(r, sizeof(r), "%08d", rank);
    return cycle_dir(folder, cycle) + "/checkpoint_cycle_" + std::to_string(cycle) + "." + r + ".chk";
}

std::string meta_name(const char *folder, int cycle) {
    return cycle_dir(folder, cycle) + "/checkpoint_cycle_" + std::to_string(cycle) + ".json";
}

std::string collection(int dim, int order) {
    return "L2_T1_" + std::to_string(dim) + "D_P" + std::to_string(order);
}

// -------------------------------------------------------- GL -> equispaced
std::vector<double> gl_nodes(int N) {   // Gauss-Lobatto nodes on [0, 1]
    std::vector<double> xi(N + 1);
    for (int i = 0; i <= N; ++i) {
        long double x = -std::cos((long double)M_PI * i / N);
        if (i > 0 && i < N)
            for (int it = 0; it < 100; ++it) {
                long double p0 = 1, p1 = x, d0 = 0, d1 = 1;
                for (int k = 1; k < N; ++k) {
                    const long double p2 = ((2 * k + 1) * x * p1 - k * p0) / (k + 1);
                    const long double d2 = d0 + (2 * k + 1) * p1;
                    p0 = p1, p1 = p2, d0 = d1, d1 = d2;
                }
                const long double dx = (1 - x * x) * d1 / (-(long double)(N * (N + 1)) * p1);
                x -= dx;
                if (std::fabs((double)dx) < 1e-30) break;
            }
        xi[i] = i == 0 ? 0.0 : i == N ? 1.0 : (double)((x + 1) * 0.5L);
    }
    return xi;
}

// L[a][l]: Lagrange basis l of the GL nodes at equispaced point a / N
std::vector<double> gl_to_equispaced(int N) {
    const std::vector<double> x = gl_nodes(N);
    std::vector<double> L((size_t)(N + 1) * (N + 1));
    for (int a = 0; a <= N; ++a) {
        const double t = (double)a / N;
        for (int l = 0; l <= N; ++l) {
            double v = 1.0;
            for (int m = 0; m <= N; ++m)
                if (m != l) v *= (t - x[m]) / (x[l] - x[m]);
            L[(size_t)a * (N + 1) + l] = v;
        }
    }
    return L;
}

// VTK Lagrange cell point index of lattice point (i, j[, k]) of an order-N
// quadrilateral / hexahedron: corners, then edge interiors, face interiors,
// cell interior, as VTK's higher-order cells number them.
int vtk_quad_index(int i, int j, int N) {
    const bool ib = i == 0 || i == N, jb = j == 0 || j == N;
    if (ib && jb) return i ? (j ? 2 : 1) : (j ? 3 : 0);
    int off = 4;
    if (!ib && jb) return off + (i - 1) + (j ? 2 * (N - 1) : 0);
    if (ib && !jb) return off + (j - 1) + (i ? N - 1 : 3 * (N - 1));
    off += 4 * (N - 1);
    return off + (i - 1) + (N - 1) * (j - 1);
}

int vtk_hex_index(int i, int j, int k, int N) {
    const bool ib = i == 0 || i == N, jb = j == 0 || j == N, kb = k == 0 || k == N;
    const int nb = ib + jb + kb, M = N - 1;
    if (nb == 3) return (i ? (j ? 2 : 1) : (j ? 3 : 0)) + (k ? 4 : 0);
    int off = 8;
    if (nb == 2) {   // edges: 4 along i / j at k = 0, the same at k = N, then 4 along k
        if (!ib) return off + (i - 1) + (j ? 2 * M : 0) + (k ? 4 * M : 0);
        if (!jb) return off + (j - 1) + (i ? M : 3 * M) + (k ? 4 * M : 0);
        off += 8 * M;
        return off + (k - 1) + M * (i ? (j ? 3 : 1) : (j ? 2 : 0));
    }
    off += 12 * M;
    if (nb == 1) {   // faces: i = 0, N; j = 0, N; k = 0, N
        if (ib) return off + (j - 1) + M * (k - 1) + (i ? M * M : 0);
        off += 2 * M * M;
        if (jb) return off + (i - 1) + M * (k - 1) + (j ? M * M : 0);
        off += 2 * M * M;
        return off + (i - 1) + M * (j - 1) + (k ? M * M : 0);
    }
    off += 6 * M * M;
    return off + (i - 1) + M * ((j - 1) + M * (k - 1));
}

const char kB64[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";

std::string base64(const unsigned char *p, size_t n) {
    std::string out;
    out.reserve((n + 2) / 3 * 4);
    for (size_t i = 0; i < n; i += 3) {
        const uint32_t v = (uint32_t)p[i] << 16 | (i + 1 < n ? (uint32_t)p[i + 1] << 8 : 0u) | (i + 2 < n ? p[i + 2] : 0u);
        out += kB64[(v >> 18) & 63];
        out += kB64[(v >> 12) & 63];
        out += i + 1 < n ? kB64[(v >> 6) & 63] : '=';
        out += i + 2 < n ? kB64[v & 63] : '=';
    }
    return out;
}

// one DataArray: binary = base64 of (uint32 byte count, raw little-endian data)
template <typename T>
void data_array(std::ostream &os, const char *type, const char *name, int ncomp, const std::vector<T> &v,
                bool binary) {
    os << "<DataArray type=\"" << type << "\" Name=\"" << name << "\" NumberOfComponents=\"" << ncomp
       << "\" format=\"" << (binary ? "binary" : "ascii") << "\">\n";
    if (binary) {
        const uint32_t nb = (uint32_t)(v.size() * sizeof(T));
        std::vector<unsigned char> buf(sizeof(uint32_t) + nb);
        std::memcpy(buf.data(), &nb, sizeof(uint32_t));
        if (nb) std::memcpy(buf.data() + sizeof(uint32_t), v.data(), nb);
        os << base64(buf.data(), buf.size()) << "\n";
    } else {
        char tmp[32];
        for (size_t i = 0; i < v.size(); ++i) {
            if (sizeof(T) == 8 && std::strcmp(type, "Float64") == 0) std::snprintf(tmp, sizeof(tmp), "%.17g", (double)v[i]);
            else std::snprintf(tmp, sizeof(tmp), "%lld", (long long)v[i]);
            os << tmp << ((i + 1) % 8 == 0 ? "\n" : " ");
        }
        os << "\n";
    }
    os << "</DataArray>\n";
}

}   // namespace

extern "C" {

prandtl_status prandtl_checkpoint_save(const char *folder, int cycle, double time, int rank, int dim, int order,
                                       long long ndof, const double *u) {
    if (!folder || !u || dim < 2 || dim > 3 || order < 1 || ndof <= 0 || rank < 0 || cycle < 0)
        return io_fail(PRANDTL_EINVAL, "bad checkpoint arguments");
    const std::string dir = cycle_dir(folder, cycle);
    if (!make_dirs(dir)) return io_fail(PRANDTL_EINVAL, "cannot create " + dir);
    {
        std::FILE *f = std::fopen(chk_name(folder, cycle, rank).c_str(), "wb");
        if (!f) return io_fail(PRANDTL_EINVAL, "cannot write " + chk_name(folder, cycle, rank));
        std::fprintf(f, "FiniteElementSpace\nFiniteElementCollection: %s\nVDim: %d\nOrdering: 0\n\n",
                     collection(dim, order).c_str(), dim + 2);
        const long long n = ndof * (dim + 2);
        for (long long i = 0; i < n; ++i) std::fprintf(f, "%.17g\n", u[i]);
        if (std::fclose(f) != 0) return io_fail(PRANDTL_EINVAL, "write failed");
    }
    if (rank == 0) {
        std::FILE *f = std::fopen(meta_name(folder, cycle).c_str(), "w");
        if (!f) return io_fail(PRANDTL_EINVAL, "cannot write " + meta_name(folder, cycle));
        std::fprintf(f, "{\n \"time\": %.17g,\n \"cycle\": %d\n}\n", time, cycle);
        if (std::fclose(f) != 0) return io_fail(PRANDTL_EINVAL, "write failed");
    }
    return PRANDTL_OK;
}

prandtl_status prandtl_checkpoint_load(const char *folder, int cycle, int rank, int dim, int order, long long ndof,
                                       double *u, double *time) {
    if (!folder || !u || dim < 2 || dim > 3 || order < 1 || ndof <= 0 || rank < 0 || cycle <= 0)
        return io_fail(PRANDTL_EINVAL, "bad checkpoint arguments (cycle must be > 0, as the reference requires)");
    {   // meta: {"time": t, "cycle": ti}
        std::ifstream m(meta_name(folder, cycle));
        if (!m) return io_fail(PRANDTL_EINVAL, "cannot open " + meta_name(folder, cycle));
        std::stringstream ss;
        ss << m.rdbuf();
        const std::string s = ss.str();
        auto number = [&](const char *key, double &out) {
            const size_t k = s.find(std::string("\"") + key + "\"");
            if (k == std::string::npos) return false;
            const size_t c = s.find(':', k);
            if (c == std::string::npos) return false;
            char *end = nullptr;
            out = std::strtod(s.c_str() + c + 1, &end);
            return end != s.c_str() + c + 1;
        };
        double t = 0.0, cyc = 0.0;
        if (!number("time", t)) t = 0.0;
        if (!number("cycle", cyc)) cyc = 0.0;
        if ((int)cyc != cycle) return io_fail(PRANDTL_EINVAL, "cycle in the meta file does not match the requested cycle");
        if (time) *time = t;
    }
    std::ifstream f(chk_name(folder, cycle, rank));
    if (!f) return io_fail(PRANDTL_EINVAL, "cannot open " + chk_name(folder, cycle, rank));
    std::string tok, coll;
    int vdim = 0, ordering = 0;
    f >> tok;
    if (tok != "FiniteElementSpace") return io_fail(PRANDTL_EINVAL, "not an MFEM GridFunction");
    f >> tok >> coll >> tok >> vdim >> tok >> ordering;
    if (coll != collection(dim, order) || vdim != dim + 2)
        return io_fail(PRANDTL_EINVAL, "checkpoint holds " + coll + " with VDim " + std::to_string(vdim) +
                                           ", expected " + collection(dim, order) + " with VDim " +
                                           std::to_string(dim + 2));
    const long long n = ndof * (dim + 2);
    std::vector<double> v(n);
    for (long long i = 0; i < n; ++i)
        if (!(f >> v[i])) return io_fail(PRANDTL_EINVAL, "checkpoint shorter than the state");
    if (ordering == 0) std::memcpy(u, v.data(), sizeof(double) * n);
    else
        for (long long i = 0; i < ndof; ++i)
            for (int c = 0; c < dim + 2; ++c) u[c * ndof + i] = v[i * (dim + 2) + c];
    return PRANDTL_OK;
}

prandtl_status prandtl_paraview_save(const char *dir, const char *name, int cycle, double time, int dim, int order,
                                     int num_elements, const double *coords, const double *u, const double *alpha,
                                     double gamma, int binary) {
    if (!dir || !name || !coords || !u || dim < 2 || dim > 3 || order < 1 || num_elements <= 0 || cycle < 0)
        return io_fail(PRANDTL_EINVAL, "bad ParaView arguments");
    const int Np = order + 1, N = order;
    const long long ND = dim == 2 ? Np * Np : Np * Np * Np, E = num_elements, Ndof = E * ND;
    const std::string root = std::string(dir) + "/" + name;
    char cyc[32];
    std::snprintf(cyc, sizeof(cyc), "Cycle%06d", cycle);
    const std::string cdir = root + "/" + cyc;
    if (!make_dirs(cdir)) return io_fail(PRANDTL_EINVAL, "cannot create " + cdir);

    // fields at the nodes, then interpolated to the cells' equispaced lattice
    const int nfld = dim + 3;   // rho, u, v, (w), p, alpha
    std::vector<double> node(Ndof * (nfld + dim));
    for (long long n = 0; n < Ndof; ++n) {
        const double rho = u[n];
        double vv = 0.0;
        for (int d = 0; d < dim; ++d) {
            const double vd = u[(1 + d) * Ndof + n] / rho;
            node[(1 + d) * Ndof + n] = vd;
            vv += vd * vd;
        }
        node[n] = rho;
        node[(1 + dim) * Ndof + n] = (gamma - 1.0) * (u[(dim + 1) * Ndof + n] - 0.5 * rho * vv);
        node[(2 + dim) * Ndof + n] = alpha ? alpha[n / ND] : 0.0;
        for (int d = 0; d < dim; ++d) node[(nfld + d) * Ndof + n] = coords[d * Ndof + n];
    }
    const std::vector<double> L = gl_to_equispaced(N);
    const int nq = nfld + dim;
    std::vector<double> pts(Ndof * 3, 0.0), fld((size_t)nfld * Ndof);
    for (long long e = 0; e < E; ++e)
        for (int q = 0; q < nq; ++q) {
            const double *src = &node[q * Ndof + e * ND];
            // tensor-product interpolation, one direction at a time
            std::vector<double> a(src, src + ND), b(ND);
            for (int r = 0; r < dim; ++r) {
                const int stride = r == 0 ? 1 : r == 1 ? Np : Np * Np;
                for (long long n = 0; n < ND; ++n) {
                    const int c = (int)((n / stride) % Np);
                    const long long base = n - (long long)c * stride;
                    double s = 0.0;
                    for (int l = 0; l < Np; ++l) s += L[(size_t)c * Np + l] * a[base + (long long)l * stride];
                    b[n] = s;
                }
                a.swap(b);
            }
            for (long long n = 0; n < ND; ++n) {
                const int i = (int)(n % Np), j = (int)((n / Np) % Np), k = (int)(n / (Np * Np));
                const long long p = e * ND + (dim == 2 ? vtk_quad_index(i, j, N) : vtk_hex_index(i, j, k, N));
                if (q < nfld) fld[(size_t)q * Ndof + p] = a[n];
                else pts[p * 3 + (q - nfld)] = a[n];
            }
        }
    std::vector<int64_t> conn(Ndof), offs(E);
    std::vector<uint8_t> types(E, (uint8_t)(dim == 2 ? 70 : 72));   // VTK_LAGRANGE_QUADRILATERAL / _HEXAHEDRON
    for (long long i = 0; i < Ndof; ++i) conn[i] = i;
    for (long long e = 0; e < E; ++e) offs[e] = (e + 1) * ND;
    const char *names[] = {"Density", "Horizontal V", "Vertical V", "Normal V"};
    {
        std::ofstream os(cdir + "/proc000000.vtu");
        if (!os) return io_fail(PRANDTL_EINVAL, "cannot write " + cdir + "/proc000000.vtu");
        os << "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\" "
              "header_type=\"UInt32\">\n<UnstructuredGrid>\n<Piece NumberOfPoints=\""
           << Ndof << "\" NumberOfCells=\"" << E << "\">\n<Points>\n";
        data_array(os, "Float64", "Points", 3, pts, binary != 0);
        os << "</Points>\n<Cells>\n";
        data_array(os, "Int64", "connectivity", 1, conn, binary != 0);
        data_array(os, "Int64", "offsets", 1, offs, binary != 0);
        data_array(os, "UInt8", "types", 1, types, binary != 0);
        os << "</Cells>\n<PointData>\n";
        for (int q = 0; q < nfld; ++q) {
            std::vector<double> col(fld.begin() + (size_t)q * Ndof, fld.begin() + (size_t)(q + 1) * Ndof);
            const char *nm = q <= dim ? names[q] : q == dim + 1 ? "Pressure" : "Blending Coeff";
            data_array(os, "Float64", nm, 1, col, binary != 0);
        }
        os << "</PointData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n";
        if (!os) return io_fail(PRANDTL_EINVAL, "write failed");
    }
    {
        std::ofstream os(cdir + "/data.pvtu");
        os << "<?xml version=\"1.0\"?>\n<VTKFile type=\"PUnstructuredGrid\" version=\"0.1\" "
              "byte_order=\"LittleEndian\" header_type=\"UInt32\">\n<PUnstructuredGrid GhostLevel=\"0\">\n"
              "<PPoints><PDataArray type=\"Float64\" Name=\"Points\" NumberOfComponents=\"3\"/></PPoints>\n<PPointData>\n";
        for (int q = 0; q < nfld; ++q) {
            const char *nm = q <= dim ? names[q] : q == dim + 1 ? "Pressure" : "Blending Coeff";
            os << "<PDataArray type=\"Float64\" Name=\"" << nm << "\" NumberOfComponents=\"1\"/>\n";
        }
        os << "</PPointData>\n<Piece Source=\"proc000000.vtu\"/>\n</PUnstructuredGrid>\n</VTKFile>\n";
    }
    // collection file: earlier cycles kept, this one replaced or appended
    const std::string pvd = root + "/" + name + ".pvd";
    std::vector<std::string> entries;
    {
        std::ifstream in(pvd);
        std::string line;
        const std::string mine = std::string("file=\"") + cyc + "/data.pvtu\"";
        while (std::getline(in, line))
            if (line.find("<DataSet") != std::string::npos && line.find(mine) == std::string::npos) entries.push_back(line);
    }
    char ent[512];
    std::snprintf(ent, sizeof(ent), "<DataSet timestep=\"%.17g\" group=\"\" part=\"0\" file=\"%s/data.pvtu\"/>", time,
                  cyc);
    entries.push_back(ent);
    std::ofstream os(pvd);
    os << "<?xml version=\"1.0\"?>\n<VTKFile type=\"Collection\" version=\"0.1\" byte_order=\"LittleEndian\">\n<Collection>\n";
    for (const auto &l : entries) os << l << "\n";
    os << "</Collection>\n</VTKFile>\n";
    if (!os) return io_fail(PRANDTL_EINVAL, "cannot write " + pvd);
    return PRANDTL_OK;
}

const char *prandtl_io_last_error(void) { return g_io_error.c_str(); }

}   // extern "C"
