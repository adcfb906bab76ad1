// Mesh ingestion: MFEM v1.0 (".mesh") and Gmsh 2.2 ASCII (".msh") meshes of
// quadrilaterals / hexahedra, into the descriptor prandtl_create takes.
//
// The reference reads its meshes through MFEM (Simulation.cpp:271-336:
// `new Mesh(file)`, `UniformRefinement()` per `ser_ref_levels`,
// `GetHilbertElementOrdering` + `ReorderElements` for "mesh_ordering":
// "Hilbert") and hands the DGSEM operator the element transformations and
// face transformations.  The kernels need, per element, the affine Jacobian's
// adjugate and determinant, and per face the two elements with aligned local
// faces (2*dir + side) and the outward scaled normal.  This file builds that:
//
//  * parsing: MFEM v1.0 elements / boundary / vertices, optionally with a
//    `nodes` section of L2_T1_*_P1 corner nodes (how MFEM stores periodic
//    meshes: identified vertices for the topology, per-element corners for the
//    geometry); Gmsh 2.2 ASCII $PhysicalNames / $Nodes / $Elements.
//  * orientation: every element's local frame is chosen (a signed permutation
//    of its reference axes) so that across each interior face the neighbour's
//    frame is aligned: face 2d+1 of one element meets face 2d of the other with
//    the same tangential axes.  A breadth-first walk fixes each neighbour's
//    frame from the shared face's vertex ids; meshes without such a frame (not
//    structured-topology) are rejected.
//  * geometry: affine elements (parallelograms / parallelepipeds) give one
//    adjugate and determinant per element; any other quadrilateral /
//    hexahedron is the multilinear map of its corners (MFEM's order-1
//    transformation), evaluated at every Gauss-Lobatto node.  The scaled face
//    normal is the signed adjugate row of the face direction (Nanson), per
//    face or, on multilinear elements, per face node: what MFEM's CalcOrtho
//    returns there.
//  * uniform refinement (2^dim children per element, the aligned frames carry
//    over) and Hilbert-curve element ordering of the element centroids.
//
// Elem1 of an interior face is the lower-numbered element (for a self-adjacent
// element, the lower local face), as MFEM's face generation assigns it when
// elements are visited in order.  Host code only.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/prandtl_b200.h"

struct prandtl_mesh {
    int dim = 0, order = 0;
    // oriented affine elements: x = X0 + J xi, xi in [0,1]^dim
    std::vector<double> X0, J;   // [E][dim], [E][dim][dim] with J[i][r] = dx_i / dxi_r
    // multilinear elements (some element is not affine): the oriented corners
    // [E][2^dim][dim], corner b at reference vertex (b & 1, b >> 1 & 1, b >> 2 & 1)
    bool multilinear = false;
    std::vector<double> Xc;
    std::vector<double> nadj, ndetj, fnn;   // descriptor per-node arrays (multilinear)
    std::vector<int> attr;       // element attributes
    // neighbour of local face lf = 2d+s: element (or -1) and its local face, or
    // the boundary attribute (0 = a boundary face no boundary element names)
    std::vector<int> nb_e, nb_f;   // [E][2*dim]
    std::map<std::pair<int, int>, std::string> names;   // (entity dim, attribute) -> name
    // descriptor arrays
    std::vector<double> adj, detj, nor;
    std::vector<int> faces, face_attr;
    double hmin = 0.0;
};

namespace {

thread_local std::string g_mesh_error;

prandtl_status mesh_fail(prandtl_status st, const std::string &msg) {
    g_mesh_error = msg;
    return st;
}

struct Raw {
    int dim = 0;
    int sdim = 0;
    std::vector<double> vx;                   // [nv][sdim]
    std::vector<std::vector<int>> el, bdr;    // corner vertex ids in lexicographic corner order
    std::vector<int> el_attr, bdr_attr;
    std::vector<double> corners;              // optional [E][2^dim][dim] (MFEM nodes section)
    std::map<std::pair<int, int>, std::string> names;
};

// lexicographic corner (bit r = coordinate along axis r) -> MFEM / Gmsh vertex slot
constexpr int QUAD_LEX[4] = {0, 1, 3, 2};
constexpr int HEX_LEX[8] = {0, 1, 3, 2, 4, 5, 7, 6};

std::vector<int> lex_corners(const std::vector<int> &v, int dim) {
    std::vector<int> c(1u << dim);
    for (size_t b = 0; b < c.size(); ++b) c[b] = v[dim == 2 ? QUAD_LEX[b] : HEX_LEX[b]];
    return c;
}

// ------------------------------------------------------------------ MFEM v1.0
std::string strip_comments(std::istream &in) {
    std::string out, line;
    while (std::getline(in, line)) {
        const size_t h = line.find('#');
        if (h != std::string::npos) line.resize(h);
        out += line;
        out += '\n';
    }
    return out;
}

prandtl_status read_mfem(std::istream &file, Raw &R) {
    std::istringstream in(strip_comments(file));
    std::string tok, a, b;
    in >> a >> b >> tok;
    if (a != "MFEM" || b != "mesh" || (tok != "v1.0" && tok != "v1.1"))
        return mesh_fail(PRANDTL_EUNSUPPORTED, "not an MFEM v1.0 mesh");
    int nv = -1;
    bool have_coords = false;
    while (in >> tok) {
        if (tok == "dimension") {
            in >> R.dim;
            if (R.dim != 2 && R.dim != 3) return mesh_fail(PRANDTL_EUNSUPPORTED, "dimension must be 2 or 3");
        } else if (tok == "elements" || tok == "boundary") {
            const bool volume = tok == "elements";
            int n = 0;
            in >> n;
            for (int k = 0; k < n && in; ++k) {
                int at = 0, geom = 0;
                in >> at >> geom;
                const int want = volume ? (R.dim == 2 ? 3 : 5) : (R.dim == 2 ? 1 : 3);
                const int nvert = geom == 1 ? 2 : geom == 3 ? 4 : geom == 5 ? 8 : geom == 2 ? 3 : geom == 4 ? 4 : 0;
                if (geom != want)
                    return mesh_fail(PRANDTL_EUNSUPPORTED, std::string(volume ? "element" : "boundary element") +
                                                               " of geometry type " + std::to_string(geom) +
                                                               ": only quadrilaterals / hexahedra are supported");
                std::vector<int> v(nvert);
                for (int &x : v) in >> x;
                if (volume) {
                    R.el.push_back(lex_corners(v, R.dim));
                    R.el_attr.push_back(at);
                } else {
                    if (R.dim == 3) v = lex_corners(v, 2);
                    R.bdr.push_back(v);
                    R.bdr_attr.push_back(at);
                }
            }
        } else if (tok == "vertices") {
            in >> nv;
            std::streampos p = in.tellg();
            std::string next;
            in >> next;
            if (next == "nodes") {   // geometry from the nodes section below
                in.seekg(p);
                continue;
            }
            R.sdim = std::atoi(next.c_str());
            if (R.sdim < R.dim) return mesh_fail(PRANDTL_EINVAL, "vertex dimension below the mesh dimension");
            R.vx.resize((size_t)nv * R.sdim);
            for (double &x : R.vx) in >> x;
            have_coords = true;
        } else if (tok == "nodes") {
            std::string fes, key, coll;
            int vdim = 0, ordering = 0;
            in >> fes >> key >> coll;
            in >> key >> vdim >> key >> ordering;
            const std::string want = std::string("L2_T1_") + (R.dim == 2 ? "2D" : "3D") + "_P1";
            if (coll != want)
                return mesh_fail(PRANDTL_EUNSUPPORTED, "nodes of collection " + coll + ": only " + want +
                                                           " (corner nodes of affine elements) are supported");
            if (vdim != R.dim) return mesh_fail(PRANDTL_EUNSUPPORTED, "nodes VDim must equal the dimension");
            const size_t nc = (size_t)1 << R.dim, E = R.el.size();
            std::vector<double> v(E * nc * vdim);
            for (double &x : v) in >> x;
            R.corners.assign(E * nc * R.dim, 0.0);
            for (size_t e = 0; e < E; ++e)
                for (size_t c = 0; c < nc; ++c)
                    for (int d = 0; d < R.dim; ++d)
                        R.corners[(e * nc + c) * R.dim + d] =
                            ordering == 1 ? v[(e * nc + c) * vdim + d] : v[(size_t)d * E * nc + e * nc + c];
            have_coords = true;
        } else if (tok == "mfem_mesh_end" || tok == "attribute_sets" || tok == "bdr_attribute_sets") {
            break;
        } else {
            return mesh_fail(PRANDTL_EUNSUPPORTED, "unknown MFEM mesh section '" + tok + "'");
        }
    }
    if (R.dim == 0 || R.el.empty() || !have_coords) return mesh_fail(PRANDTL_EINVAL, "incomplete MFEM mesh");
    for (const auto &v : R.el)
        for (int x : v)
            if (x < 0 || x >= nv) return mesh_fail(PRANDTL_EINVAL, "vertex index out of range");
    return PRANDTL_OK;
}

// ------------------------------------------------------------ Gmsh 2.2 ASCII
prandtl_status read_gmsh(std::istream &in, Raw &R) {
    std::string line;
    std::map<long, int> node_id;
    std::vector<double> xyz;
    struct GEl { int type, tag; std::vector<long> nodes; };
    std::vector<GEl> els;
    while (std::getline(in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line == "$MeshFormat") {
            std::getline(in, line);
            double ver = 0;
            int ft = 0;
            std::istringstream s(line);
            s >> ver >> ft;
            if (ver < 2.0 || ver >= 3.0 || ft != 0)
                return mesh_fail(PRANDTL_EUNSUPPORTED, "Gmsh format " + line + ": only 2.x ASCII is supported");
        } else if (line == "$PhysicalNames") {
            std::getline(in, line);
            const int n = std::atoi(line.c_str());
            for (int k = 0; k < n && std::getline(in, line); ++k) {
                std::istringstream s(line);
                int d = 0, tag = 0;
                s >> d >> tag;
                std::string rest;
                std::getline(s, rest);
                const size_t q0 = rest.find('"'), q1 = rest.rfind('"');
                R.names[{d, tag}] = (q0 != std::string::npos && q1 > q0) ? rest.substr(q0 + 1, q1 - q0 - 1) : rest;
            }
        } else if (line == "$Nodes") {
            std::getline(in, line);
            const long n = std::atol(line.c_str());
            xyz.reserve((size_t)n * 3);
            for (long k = 0; k < n && std::getline(in, line); ++k) {
                std::istringstream s(line);
                long id = 0;
                double x = 0, y = 0, z = 0;
                s >> id >> x >> y >> z;
                node_id[id] = (int)(xyz.size() / 3);
                xyz.push_back(x);
                xyz.push_back(y);
                xyz.push_back(z);
            }
        } else if (line == "$Elements") {
            std::getline(in, line);
            const long n = std::atol(line.c_str());
            for (long k = 0; k < n && std::getline(in, line); ++k) {
                std::istringstream s(line);
                long id = 0;
                int type = 0, ntags = 0;
                s >> id >> type >> ntags;
                std::vector<int> tags(ntags);
                for (int &t : tags) s >> t;
                GEl g{type, ntags > 0 ? tags[0] : 1, {}};
                long v;
                while (s >> v) g.nodes.push_back(v);
                els.push_back(std::move(g));
            }
        }
    }
    int dim = 0;
    for (const auto &g : els) {   // 1: 2-node line, 3: 4-node quad, 5: 8-node hex, 15: point
        if (g.type == 5) dim = 3;
        else if (g.type == 3 && dim < 2) dim = 2;
        else if (g.type != 1 && g.type != 3 && g.type != 15)
            return mesh_fail(PRANDTL_EUNSUPPORTED, "Gmsh element type " + std::to_string(g.type) +
                                                       ": only 4-node quadrilaterals / 8-node hexahedra");
    }
    if (dim == 0) return mesh_fail(PRANDTL_EINVAL, "no quadrilateral or hexahedral elements");
    R.dim = dim;
    R.sdim = 3;
    R.vx = xyz;
    const int vol_type = dim == 2 ? 3 : 5, bdr_type = dim == 2 ? 1 : 3;
    for (const auto &g : els) {
        if (g.type != vol_type && g.type != bdr_type) continue;
        std::vector<int> v;
        for (long id : g.nodes) {
            auto it = node_id.find(id);
            if (it == node_id.end()) return mesh_fail(PRANDTL_EINVAL, "element names an unknown node");
            v.push_back(it->second);
        }
        if (g.type == vol_type) {
            if ((int)v.size() != (1 << dim)) return mesh_fail(PRANDTL_EINVAL, "bad element node count");
            R.el.push_back(lex_corners(v, dim));
            R.el_attr.push_back(g.tag);
        } else {
            if ((int)v.size() != (1 << (dim - 1))) return mesh_fail(PRANDTL_EINVAL, "bad boundary node count");
            R.bdr.push_back(dim == 3 ? lex_corners(v, 2) : v);
            R.bdr_attr.push_back(g.tag);
        }
    }
    if (R.el.empty()) return mesh_fail(PRANDTL_EINVAL, "no volume elements");
    return PRANDTL_OK;
}

// --------------------------------------------------------------- orientation
// A frame: new axis r is old axis perm[r], reversed when flip bit r is set.
struct Frame {
    std::array<int, 3> perm{0, 1, 2};
    int flip = 0;
};

int old_corner(const Frame &F, int dim, int b) {
    int o = 0;
    for (int r = 0; r < dim; ++r) o |= ((((b >> r) & 1) ^ ((F.flip >> r) & 1)) << F.perm[r]);
    return o;
}

std::vector<Frame> all_frames(int dim) {
    std::vector<Frame> out;
    std::array<int, 3> p{0, 1, 2};
    do {
        if (dim == 2 && p[2] != 2) continue;
        for (int f = 0; f < (1 << dim); ++f) {
            Frame F;
            F.perm = p;
            F.flip = f;
            out.push_back(F);
        }
    } while (std::next_permutation(p.begin(), p.begin() + dim));
    return out;
}

// corners of local face (d, s) in tangential lexicographic order
std::vector<int> face_corner_bits(int dim, int d, int s) {
    std::vector<int> out;
    for (int b = 0; b < (1 << dim); ++b)
        if (((b >> d) & 1) == s) out.push_back(b);
    return out;   // increasing b = lexicographic in the remaining axes
}

uint64_t face_key(std::vector<int> ids) {
    std::sort(ids.begin(), ids.end());
    uint64_t h = 1469598103934665603ull;
    for (int x : ids) h = (h ^ (uint64_t)(uint32_t)x) * 1099511628211ull;
    return h;
}

void adjugate(int dim, const double *J, double *A) {   // A = adj(J), J row-major J[i][r]
    if (dim == 2) {
        A[0] = J[3];
        A[1] = -J[1];
        A[2] = -J[2];
        A[3] = J[0];
        return;
    }
    A[0] = J[4] * J[8] - J[5] * J[7];
    A[1] = J[2] * J[7] - J[1] * J[8];
    A[2] = J[1] * J[5] - J[2] * J[4];
    A[3] = J[5] * J[6] - J[3] * J[8];
    A[4] = J[0] * J[8] - J[2] * J[6];
    A[5] = J[2] * J[3] - J[0] * J[5];
    A[6] = J[3] * J[7] - J[4] * J[6];
    A[7] = J[1] * J[6] - J[0] * J[7];
    A[8] = J[0] * J[4] - J[1] * J[3];
}

double determinant(int dim, const double *J) {
    if (dim == 2) return J[0] * J[3] - J[1] * J[2];
    return J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
           J[2] * (J[3] * J[7] - J[4] * J[6]);
}

// smallest singular value of J (MFEM GetElementSize(e, 1)): sqrt of the
// smallest eigenvalue of J^T J (closed form in 2D, Jacobi sweeps in 3D)
double min_singular(int dim, const double *J) {
    double G[9] = {0};
    for (int a = 0; a < dim; ++a)
        for (int b = 0; b < dim; ++b)
            for (int i = 0; i < dim; ++i) G[a * dim + b] += J[i * dim + a] * J[i * dim + b];
    if (dim == 2) {
        const double t = 0.5 * (G[0] + G[3]), d = std::sqrt(std::max(0.0, 0.25 * (G[0] - G[3]) * (G[0] - G[3]) + G[1] * G[2]));
        return std::sqrt(std::max(0.0, t - d));
    }
    for (int sweep = 0; sweep < 50; ++sweep) {
        double off = std::fabs(G[1]) + std::fabs(G[2]) + std::fabs(G[5]);
        if (off < 1e-300) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                const double apq = G[p * 3 + q];
                if (std::fabs(apq) < 1e-300) continue;
                const double th = 0.5 * (G[q * 3 + q] - G[p * 3 + p]) / apq;
                const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {   // G = R^T G R
                    const double gkp = G[k * 3 + p], gkq = G[k * 3 + q];
                    G[k * 3 + p] = c * gkp - s * gkq;
                    G[k * 3 + q] = s * gkp + c * gkq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double gpk = G[p * 3 + k], gqk = G[q * 3 + k];
                    G[p * 3 + k] = c * gpk - s * gqk;
                    G[q * 3 + k] = s * gpk + c * gqk;
                }
            }
    }
    return std::sqrt(std::max(0.0, std::min(G[0], std::min(G[4], G[8]))));
}

prandtl_status orient(const Raw &R, prandtl_mesh &M) {
    const int dim = R.dim, nc = 1 << dim, nfl = 2 * dim;
    const int E = (int)R.el.size();
    for (int e = 0; e < E; ++e) {
        std::vector<int> v = R.el[e];
        std::sort(v.begin(), v.end());
        if (std::adjacent_find(v.begin(), v.end()) != v.end())
            return mesh_fail(PRANDTL_EUNSUPPORTED, "element " + std::to_string(e) +
                                                       " repeats a vertex (a periodic direction one element wide)");
    }
    // faces of the original frames, by vertex set
    std::multimap<uint64_t, std::pair<int, std::vector<int>>> fmap;
    for (int e = 0; e < E; ++e)
        for (int lf = 0; lf < nfl; ++lf) {
            std::vector<int> ids;
            for (int b : face_corner_bits(dim, lf >> 1, lf & 1)) ids.push_back(R.el[e][b]);
            std::vector<int> key = ids;
            std::sort(key.begin(), key.end());
            fmap.emplace(face_key(key), std::make_pair(e, key));
        }
    std::map<uint64_t, int> battr;
    for (size_t k = 0; k < R.bdr.size(); ++k) battr[face_key(R.bdr[k])] = R.bdr_attr[k];

    const std::vector<Frame> frames = all_frames(dim);
    std::vector<int> fr(E, -1);
    M.nb_e.assign((size_t)E * nfl, -2);
    M.nb_f.assign((size_t)E * nfl, 0);
    auto corner_ids = [&](int e, const Frame &F, int lf) {
        std::vector<int> ids;
        for (int b : face_corner_bits(dim, lf >> 1, lf & 1)) ids.push_back(R.el[e][old_corner(F, dim, b)]);
        return ids;
    };
    auto corner_x = [&](int e, const Frame &F, int b, int i) {
        const int o = old_corner(F, dim, b);
        return R.corners.empty() ? R.vx[(size_t)R.el[e][o] * R.sdim + i] : R.corners[((size_t)e * nc + o) * dim + i];
    };
    std::vector<int> queue;
    for (int seed = 0; seed < E; ++seed) {
        if (fr[seed] >= 0) continue;
        // the first frame with a positive Jacobian (clockwise-listed elements get
        // a reflected one); the walk carries it to the seed's component
        fr[seed] = 0;
        for (size_t k = 0; k < frames.size(); ++k) {
            double J[9];
            for (int r = 0; r < dim; ++r)
                for (int i = 0; i < dim; ++i)
                    J[i * dim + r] = corner_x(seed, frames[k], 1 << r, i) - corner_x(seed, frames[k], 0, i);
            if (determinant(dim, J) > 0.0) {
                fr[seed] = (int)k;
                break;
            }
        }
        queue.assign(1, seed);
        for (size_t qi = 0; qi < queue.size(); ++qi) {
            const int e = queue[qi];
            const Frame &Fe = frames[fr[e]];
            for (int lf = 0; lf < nfl; ++lf) {
                const std::vector<int> ids = corner_ids(e, Fe, lf);
                std::vector<int> key = ids;
                std::sort(key.begin(), key.end());
                const uint64_t h = face_key(key);
                int n = -1;
                int count = 0;
                for (auto it = fmap.lower_bound(h); it != fmap.upper_bound(h); ++it) {
                    if (it->second.second != key) continue;
                    ++count;
                    if (it->second.first != e) n = it->second.first;
                }
                if (count > 2) return mesh_fail(PRANDTL_EINVAL, "a face shared by more than two elements");
                if (count == 1) {   // boundary face
                    auto b = battr.find(h);
                    M.nb_e[(size_t)e * nfl + lf] = -1;
                    M.nb_f[(size_t)e * nfl + lf] = b == battr.end() ? 0 : b->second;
                    continue;
                }
                if (n < 0) return mesh_fail(PRANDTL_EINVAL, "element " + std::to_string(e) + " meets itself");
                const int lfn = lf ^ 1;
                if (fr[n] < 0) {
                    int pick = -1;
                    for (size_t k = 0; k < frames.size(); ++k)
                        if (corner_ids(n, frames[k], lfn) == ids) {
                            if (pick >= 0) return mesh_fail(PRANDTL_EINVAL, "ambiguous face alignment");
                            pick = (int)k;
                        }
                    if (pick < 0) return mesh_fail(PRANDTL_EINVAL, "faces cannot be matched");
                    fr[n] = pick;
                    queue.push_back(n);
                } else if (corner_ids(n, frames[fr[n]], lfn) != ids) {
                    return mesh_fail(PRANDTL_EUNSUPPORTED,
                                     "elements " + std::to_string(e) + " and " + std::to_string(n) +
                                         " admit no aligned local frames: only meshes of structured topology "
                                         "(every interior face joins faces 2d+1 and 2d with aligned traces)");
                }
                M.nb_e[(size_t)e * nfl + lf] = n;
                M.nb_f[(size_t)e * nfl + lf] = lfn;
            }
        }
    }
    // geometry in the chosen frames: X0 + J xi from corners 0 and 1 << r, and
    // the corners themselves for the multilinear map when any element is not
    // a parallelogram / parallelepiped
    M.X0.assign((size_t)E * dim, 0.0);
    M.J.assign((size_t)E * dim * dim, 0.0);
    M.Xc.assign((size_t)E * nc * dim, 0.0);
    M.multilinear = false;
    for (int e = 0; e < E; ++e) {
        const Frame &F = frames[fr[e]];
        auto X = [&](int b, int i) { return corner_x(e, F, b, i); };
        double *x0 = &M.X0[(size_t)e * dim], *J = &M.J[(size_t)e * dim * dim];
        double scale = 0.0;
        for (int i = 0; i < dim; ++i) x0[i] = X(0, i);
        for (int r = 0; r < dim; ++r)
            for (int i = 0; i < dim; ++i) {
                J[i * dim + r] = X(1 << r, i) - x0[i];
                scale = std::max(scale, std::fabs(J[i * dim + r]));
            }
        for (int b = 0; b < nc; ++b)
            for (int i = 0; i < dim; ++i) {
                M.Xc[((size_t)e * nc + b) * dim + i] = X(b, i);
                double x = x0[i];
                for (int r = 0; r < dim; ++r) x += ((b >> r) & 1) * J[i * dim + r];
                if (std::fabs(x - X(b, i)) > 1e-9 * scale) M.multilinear = true;
            }
        if (!(determinant(dim, J) > 0.0))
            return mesh_fail(PRANDTL_EINVAL, "element " + std::to_string(e) + " is inverted");
    }
    M.attr = R.el_attr;
    return PRANDTL_OK;
}

// Multilinear map of corners Xc (2^dim of them) at reference point xi: the
// position x and the Jacobian J[i][r] = dx_i / dxi_r (MFEM's order-1 H1
// transformation of a quadrilateral / hexahedron).
void multilinear_eval(int dim, const double *Xc, const double *xi, double *x, double *J) {
    const int nc = 1 << dim;
    for (int i = 0; i < dim; ++i) {
        if (x) x[i] = 0.0;
        if (J)
            for (int r = 0; r < dim; ++r) J[i * dim + r] = 0.0;
    }
    for (int b = 0; b < nc; ++b) {
        double phi = 1.0;
        for (int q = 0; q < dim; ++q) phi *= ((b >> q) & 1) ? xi[q] : 1.0 - xi[q];
        for (int i = 0; i < dim; ++i)
            if (x) x[i] += phi * Xc[b * dim + i];
        if (!J) continue;
        for (int r = 0; r < dim; ++r) {
            double dphi = ((b >> r) & 1) ? 1.0 : -1.0;
            for (int q = 0; q < dim; ++q)
                if (q != r) dphi *= ((b >> q) & 1) ? xi[q] : 1.0 - xi[q];
            for (int i = 0; i < dim; ++i) J[i * dim + r] += dphi * Xc[b * dim + i];
        }
    }
}

// Gauss-Lobatto nodes on [0, 1]: roots of (1 - x^2) P'_N (Newton in long double).
std::vector<double> gl_nodes(int N) {
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

// one level of uniform refinement: child c of element e has bits c along the
// (aligned) local axes, x = X0 + J (c + xi) / 2
void refine(prandtl_mesh &M) {
    const int dim = M.dim, nch = 1 << dim, nfl = 2 * dim;
    const int E = (int)M.attr.size();
    prandtl_mesh C;
    C.dim = dim;
    C.X0.resize((size_t)E * nch * dim);
    C.J.resize((size_t)E * nch * dim * dim);
    C.attr.resize((size_t)E * nch);
    C.nb_e.resize((size_t)E * nch * nfl);
    C.nb_f.resize((size_t)E * nch * nfl);
    for (int e = 0; e < E; ++e)
        for (int c = 0; c < nch; ++c) {
            const int ce = e * nch + c;
            C.attr[ce] = M.attr[e];
            for (int i = 0; i < dim; ++i) {
                double x = M.X0[(size_t)e * dim + i];
                for (int r = 0; r < dim; ++r) {
                    x += 0.5 * ((c >> r) & 1) * M.J[((size_t)e * dim + i) * dim + r];
                    C.J[((size_t)ce * dim + i) * dim + r] = 0.5 * M.J[((size_t)e * dim + i) * dim + r];
                }
                C.X0[(size_t)ce * dim + i] = x;
            }
            for (int lf = 0; lf < nfl; ++lf) {
                const int d = lf >> 1, s = lf & 1;
                int ne, nf;
                if (((c >> d) & 1) != s) {   // sibling
                    ne = e * nch + (c ^ (1 << d));
                    nf = lf ^ 1;
                } else if (M.nb_e[(size_t)e * nfl + lf] < 0) {   // parent boundary
                    ne = -1;
                    nf = M.nb_f[(size_t)e * nfl + lf];
                } else {   // the neighbour parent's child across the face (aligned frames)
                    ne = M.nb_e[(size_t)e * nfl + lf] * nch + (c ^ (1 << d));
                    nf = lf ^ 1;
                }
                C.nb_e[(size_t)ce * nfl + lf] = ne;
                C.nb_f[(size_t)ce * nfl + lf] = nf;
            }
        }
    if (M.multilinear) {   // child corners: the parent's map at (c + b) / 2
        const int nc = 1 << dim;
        C.Xc.resize((size_t)E * nch * nc * dim);
        for (int e = 0; e < E; ++e)
            for (int c = 0; c < nch; ++c)
                for (int b = 0; b < nc; ++b) {
                    double xi[3] = {0, 0, 0};
                    for (int r = 0; r < dim; ++r) xi[r] = 0.5 * (((c >> r) & 1) + ((b >> r) & 1));
                    multilinear_eval(dim, &M.Xc[(size_t)e * nc * dim], xi,
                                     &C.Xc[(((size_t)e * nch + c) * nc + b) * dim], nullptr);
                }
        M.Xc.swap(C.Xc);
    }
    M.X0.swap(C.X0);
    M.J.swap(C.J);
    M.attr.swap(C.attr);
    M.nb_e.swap(C.nb_e);
    M.nb_f.swap(C.nb_f);
}

// Hilbert index of integer coordinates (Skilling's transpose form, "Programming
// the Hilbert curve", AIP Conf. Proc. 707, 2004), interleaved into one key.
uint64_t hilbert_key(int dim, const uint32_t *coord, int bits) {
    uint32_t X[3] = {coord[0], coord[1], dim > 2 ? coord[2] : 0u};
    const uint32_t M = 1u << (bits - 1);
    for (uint32_t Q = M; Q > 1; Q >>= 1) {   // inverse undo
        const uint32_t P = Q - 1;
        for (int i = 0; i < dim; ++i) {
            if (X[i] & Q) X[0] ^= P;
            else {
                const uint32_t t = (X[0] ^ X[i]) & P;
                X[0] ^= t;
                X[i] ^= t;
            }
        }
    }
    for (int i = 1; i < dim; ++i) X[i] ^= X[i - 1];   // Gray encode
    uint32_t t = 0;
    for (uint32_t Q = M; Q > 1; Q >>= 1)
        if (X[dim - 1] & Q) t ^= Q - 1;
    for (int i = 0; i < dim; ++i) X[i] ^= t;
    uint64_t key = 0;
    for (int b = bits - 1; b >= 0; --b)
        for (int i = 0; i < dim; ++i) key = (key << 1) | ((X[i] >> b) & 1u);
    return key;
}

void hilbert_reorder(prandtl_mesh &M) {
    const int dim = M.dim, nfl = 2 * dim, E = (int)M.attr.size();
    const int bits = dim == 2 ? 20 : 16;
    std::vector<double> c((size_t)E * dim), lo(dim, 1e300), hi(dim, -1e300);
    const int nc = 1 << dim;
    for (int e = 0; e < E; ++e)
        for (int i = 0; i < dim; ++i) {
            double x = M.X0[(size_t)e * dim + i];
            if (M.multilinear) {   // the map at the reference centre: the corners' mean
                x = 0.0;
                for (int b = 0; b < nc; ++b) x += M.Xc[((size_t)e * nc + b) * dim + i];
                x /= nc;
            } else {
                for (int r = 0; r < dim; ++r) x += 0.5 * M.J[((size_t)e * dim + i) * dim + r];
            }
            c[(size_t)e * dim + i] = x;
            lo[i] = std::min(lo[i], x);
            hi[i] = std::max(hi[i], x);
        }
    std::vector<std::pair<uint64_t, int>> key(E);
    for (int e = 0; e < E; ++e) {
        uint32_t q[3] = {0, 0, 0};
        for (int i = 0; i < dim; ++i) {
            const double w = hi[i] > lo[i] ? (c[(size_t)e * dim + i] - lo[i]) / (hi[i] - lo[i]) : 0.0;
            q[i] = (uint32_t)std::min<double>(std::ldexp(1.0, bits) - 1, std::floor(w * std::ldexp(1.0, bits)));
        }
        key[e] = {hilbert_key(dim, q, bits), e};
    }
    std::stable_sort(key.begin(), key.end());
    std::vector<int> newof(E);
    for (int k = 0; k < E; ++k) newof[key[k].second] = k;
    prandtl_mesh C;
    C.X0.resize(M.X0.size());
    C.J.resize(M.J.size());
    C.attr.resize(E);
    C.nb_e.resize(M.nb_e.size());
    C.nb_f.resize(M.nb_f.size());
    if (M.multilinear) C.Xc.resize(M.Xc.size());
    for (int k = 0; k < E; ++k) {
        const int e = key[k].second;
        std::copy_n(&M.X0[(size_t)e * dim], dim, &C.X0[(size_t)k * dim]);
        std::copy_n(&M.J[(size_t)e * dim * dim], dim * dim, &C.J[(size_t)k * dim * dim]);
        if (M.multilinear) std::copy_n(&M.Xc[(size_t)e * nc * dim], nc * dim, &C.Xc[(size_t)k * nc * dim]);
        C.attr[k] = M.attr[e];
        for (int lf = 0; lf < nfl; ++lf) {
            const int ne = M.nb_e[(size_t)e * nfl + lf];
            C.nb_e[(size_t)k * nfl + lf] = ne < 0 ? ne : newof[ne];
            C.nb_f[(size_t)k * nfl + lf] = M.nb_f[(size_t)e * nfl + lf];
        }
    }
    if (M.multilinear) M.Xc.swap(C.Xc);
    M.X0.swap(C.X0);
    M.J.swap(C.J);
    M.attr.swap(C.attr);
    M.nb_e.swap(C.nb_e);
    M.nb_f.swap(C.nb_f);
}

// Element-local node of face node a on local face lf = 2 dir + side.
int face_node_of(int dim, int Np, int lf, int a) {
    const int d = lf >> 1, s = lf & 1;
    int c[3] = {0, 0, 0};
    c[d] = s * (Np - 1);
    if (dim == 2) {
        c[1 - d] = a;
    } else {
        const int t0 = (d == 0) ? 1 : 0, t1 = (d == 2) ? 1 : 2;
        c[t0] = a % Np;
        c[t1] = a / Np;
    }
    return c[0] + Np * (c[1] + Np * c[2]);
}

// descriptor arrays; boundary faces carry BC index attribute - 1
prandtl_status describe(prandtl_mesh &M) {
    const int dim = M.dim, nfl = 2 * dim, E = (int)M.attr.size();
    M.adj.resize((size_t)E * dim * dim);
    M.detj.resize(E);
    M.faces.clear();
    M.nor.clear();
    M.face_attr.clear();
    M.hmin = 1e300;
    const int nc = 1 << dim, Np = M.order + 1;
    int nd = 1;
    for (int d = 0; d < dim; ++d) nd *= Np;
    const int nfn = nd / Np;
    for (int e = 0; e < E; ++e) {
        double Jc[9];
        const double *J = &M.J[(size_t)e * dim * dim];
        if (M.multilinear) {   // element values at the reference centre
            const double mid[3] = {0.5, 0.5, 0.5};
            multilinear_eval(dim, &M.Xc[(size_t)e * nc * dim], mid, nullptr, Jc);
            J = Jc;
        }
        adjugate(dim, J, &M.adj[(size_t)e * dim * dim]);
        M.detj[e] = determinant(dim, J);
        M.hmin = std::min(M.hmin, min_singular(dim, J));   // MFEM GetElementSize(e, 1), at the centre
    }
    if (M.multilinear) {   // the transformation at every Gauss-Lobatto node
        const std::vector<double> xi = gl_nodes(M.order);
        M.nadj.resize((size_t)E * nd * dim * dim);
        M.ndetj.resize((size_t)E * nd);
        for (int e = 0; e < E; ++e)
            for (int n = 0; n < nd; ++n) {
                const double p[3] = {xi[n % Np], xi[(n / Np) % Np], dim > 2 ? xi[n / (Np * Np)] : 0.0};
                double J[9];
                multilinear_eval(dim, &M.Xc[(size_t)e * nc * dim], p, nullptr, J);
                adjugate(dim, J, &M.nadj[((size_t)e * nd + n) * dim * dim]);
                const double dj = determinant(dim, J);
                if (!(dj > 0.0))
                    return mesh_fail(PRANDTL_EINVAL, "element " + std::to_string(e) + " is inverted at node " +
                                                         std::to_string(n));
                M.ndetj[(size_t)e * nd + n] = dj;
            }
    }
    M.fnn.clear();
    for (int e = 0; e < E; ++e)
        for (int lf = 0; lf < nfl; ++lf) {
            const int ne = M.nb_e[(size_t)e * nfl + lf], nf = M.nb_f[(size_t)e * nfl + lf];
            if (ne >= 0 && (ne < e || (ne == e && nf < lf))) continue;   // owned by the other element
            const int d = lf >> 1;
            const double sg = (lf & 1) ? 1.0 : -1.0;
            if (ne < 0) {
                M.faces.insert(M.faces.end(), {e, lf, -1, nf - 1});
                M.face_attr.push_back(nf);
            } else {
                M.faces.insert(M.faces.end(), {e, lf, ne, nf});
                M.face_attr.push_back(0);
            }
            if (M.multilinear) {   // per face node, and their mean as the face's value
                double mean[3] = {0, 0, 0};
                for (int a = 0; a < nfn; ++a) {
                    const int n = face_node_of(dim, Np, lf, a);
                    for (int c = 0; c < dim; ++c) {
                        const double v = sg * M.nadj[(((size_t)e * nd + n) * dim + d) * dim + c];
                        M.fnn.push_back(v);
                        mean[c] += v / nfn;
                    }
                }
                for (int c = 0; c < dim; ++c) M.nor.push_back(mean[c]);
            } else {
                for (int c = 0; c < dim; ++c) M.nor.push_back(sg * M.adj[((size_t)e * dim + d) * dim + c]);
            }
        }
    return PRANDTL_OK;
}

}   // namespace

extern "C" {

prandtl_status prandtl_mesh_read(const char *path, int order, int refine_levels, int hilbert, prandtl_mesh **out) {
    if (!out) return mesh_fail(PRANDTL_EINVAL, "out is NULL");
    *out = nullptr;
    if (!path) return mesh_fail(PRANDTL_EINVAL, "path is NULL");
    if (order < 1 || order > 7) return mesh_fail(PRANDTL_EUNSUPPORTED, "order must be 1..7");
    if (refine_levels < 0 || refine_levels > 8) return mesh_fail(PRANDTL_EINVAL, "refine_levels must be 0..8");
    std::ifstream f(path);
    if (!f) return mesh_fail(PRANDTL_EINVAL, std::string("cannot open ") + path);
    Raw R;
    std::string first;
    std::getline(f, first);
    f.seekg(0);
    prandtl_status st;
    if (first.rfind("$MeshFormat", 0) == 0) st = read_gmsh(f, R);
    else if (first.rfind("MFEM mesh", 0) == 0) st = read_mfem(f, R);
    else st = mesh_fail(PRANDTL_EUNSUPPORTED, "unknown mesh format (MFEM v1.0 or Gmsh 2.2 ASCII)");
    if (st != PRANDTL_OK) return st;
    prandtl_mesh *M = new prandtl_mesh();
    M->dim = R.dim;
    M->order = order;
    M->names = R.names;
    if ((st = orient(R, *M)) != PRANDTL_OK) {
        delete M;
        return st;
    }
    const size_t E0 = M->attr.size();
    if ((E0 << (R.dim * refine_levels)) > (size_t)1 << 30) {
        delete M;
        return mesh_fail(PRANDTL_ETOOLARGE, "refined mesh above 2^30 elements");
    }
    for (int l = 0; l < refine_levels; ++l) refine(*M);
    if (hilbert) hilbert_reorder(*M);
    if ((st = describe(*M)) != PRANDTL_OK) {
        delete M;
        return st;
    }
    *out = M;
    return PRANDTL_OK;
}

prandtl_status prandtl_mesh_describe(const prandtl_mesh *m, prandtl_mesh_desc *desc, double *hmin) {
    if (!m || !desc) return mesh_fail(PRANDTL_EINVAL, "null pointer");
    desc->dim = m->dim;
    desc->order = m->order;
    desc->num_elements = (int)m->detj.size();
    desc->num_faces = (int)m->face_attr.size();
    desc->elem_adj = m->adj.data();
    desc->elem_detj = m->detj.data();
    desc->face_elems = m->faces.data();
    desc->face_nor = m->nor.data();
    desc->node_adj = m->multilinear ? m->nadj.data() : nullptr;
    desc->node_detj = m->multilinear ? m->ndetj.data() : nullptr;
    desc->face_node_nor = m->multilinear ? m->fnn.data() : nullptr;
    if (hmin) *hmin = m->hmin;
    return PRANDTL_OK;
}

prandtl_status prandtl_mesh_face_attributes(const prandtl_mesh *m, int *attr) {
    if (!m || !attr) return mesh_fail(PRANDTL_EINVAL, "null pointer");
    std::copy(m->face_attr.begin(), m->face_attr.end(), attr);
    return PRANDTL_OK;
}

prandtl_status prandtl_mesh_element_attributes(const prandtl_mesh *m, int *attr) {
    if (!m || !attr) return mesh_fail(PRANDTL_EINVAL, "null pointer");
    std::copy(m->attr.begin(), m->attr.end(), attr);
    return PRANDTL_OK;
}

prandtl_status prandtl_mesh_set_boundary_conditions(prandtl_mesh *m, const int *bc_of_attribute, int num_attributes) {
    if (!m || (num_attributes > 0 && !bc_of_attribute) || num_attributes < 0)
        return mesh_fail(PRANDTL_EINVAL, "bad boundary-condition map");
    for (size_t f = 0; f < m->face_attr.size(); ++f) {
        if (m->faces[4 * f + 2] >= 0) continue;
        const int a = m->face_attr[f];
        m->faces[4 * f + 3] = (a >= 1 && a <= num_attributes) ? bc_of_attribute[a - 1] : -1;
    }
    return PRANDTL_OK;
}

int prandtl_mesh_attribute(const prandtl_mesh *m, int entity_dim, const char *name) {
    if (!m || !name) return -1;
    for (const auto &kv : m->names)
        if (kv.first.first == entity_dim && kv.second == name) return kv.first.second;
    return -1;
}

prandtl_status prandtl_mesh_node_coords(const prandtl_mesh *m, double *xyz) {
    if (!m || !xyz) return mesh_fail(PRANDTL_EINVAL, "null pointer");
    const int dim = m->dim, Np = m->order + 1, nc = 1 << dim;
    const std::vector<double> xi = gl_nodes(m->order);
    const size_t E = m->attr.size(), ND = (size_t)std::pow(Np, dim), Ndof = E * ND;
    for (size_t e = 0; e < E; ++e)
        for (size_t n = 0; n < ND; ++n) {
            const int c[3] = {(int)(n % Np), (int)((n / Np) % Np), (int)(n / (Np * Np))};
            if (m->multilinear) {
                const double p[3] = {xi[c[0]], xi[c[1]], dim > 2 ? xi[c[2]] : 0.0};
                double x[3];
                multilinear_eval(dim, &m->Xc[e * nc * dim], p, x, nullptr);
                for (int i = 0; i < dim; ++i) xyz[(size_t)i * Ndof + e * ND + n] = x[i];
                continue;
            }
            for (int i = 0; i < dim; ++i) {
                double x = m->X0[e * dim + i];
                for (int r = 0; r < dim; ++r) x += m->J[(e * dim + i) * dim + r] * xi[c[r]];
                xyz[(size_t)i * Ndof + e * ND + n] = x;
            }
        }
    return PRANDTL_OK;
}

void prandtl_mesh_destroy(prandtl_mesh *m) { delete m; }

const char *prandtl_mesh_last_error(void) { return g_mesh_error.c_str(); }

}   // extern "C"
