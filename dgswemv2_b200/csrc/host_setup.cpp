// Host-side preprocessing of the RKDG library (see host_setup.h).
#include "host_setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>
#include <unordered_map>

#ifdef _OPENMP
#include <omp.h>
#include <parallel/algorithm>
#endif

#include "function_sets.h"
#include "quadrature.h"

namespace dgsw {

// ------------------------------------------------------------------------------------------------
// Dubiner modal basis on the master triangle (source/basis/bases_2D/basis_dubiner_2D.cpp):
// phi_(p,q) = P_p^(0,0)(n1) ((1-n2)/2)^p P_q^(2p+1,0)(n2),  n1 = 2(1+z1)/(1-z2) - 1, n2 = z2,
// with the reference's values at the collapsed vertex (-1, 1). Modes are numbered along the
// anti-diagonals p+q = 0, 1, 2, ... with q descending, matching the reference's dof -> (p,q) map.
// ------------------------------------------------------------------------------------------------
static void mode_pq(int dof, int& p, int& q) {
    int d = 0;
    while ((d + 1) * (d + 2) / 2 <= dof) ++d;  // anti-diagonal index
    p = dof - d * (d + 1) / 2;
    q = d - p;
}

// P_n^(a,b)(x) by the standard three-term recurrence
static double jacobi(int n, int a, int b, double x) {
    if (n == 0) return 1.0;
    double pm = 1.0, pc = (a - b + (a + b + 2) * x) / 2;
    for (int i = 1; i < n; ++i) {
        double c1 = 2.0 * (i + 1) * (i + a + b + 1) * (2 * i + a + b);
        double c2 = (2.0 * i + a + b + 1) * (double)(a * a - b * b);
        double c3 = (2.0 * i + a + b) * (2.0 * i + a + b + 1) * (2.0 * i + a + b + 2);
        double c4 = 2.0 * (i + a) * (i + b) * (2 * i + a + b + 2);
        double pn = ((c2 + c3 * x) * pc - c4 * pm) / c1;
        pm = pc;
        pc = pn;
    }
    return pc;
}

static double djacobi(int n, int a, int b, double x) {
    if (n == 0) return 0.0;
    if (n == 1) return (a + b + n + 1) / 2.0;
    return jacobi(n - 1, a + 1, b + 1, x) * ((a + b + n + 1) / 2.0);
}

// values at the singular vertex (-1, 1): the reference's recursions (basis_dubiner_2D.cpp:177-211)
static double sing_dz1(int q) {
    double a = 3.0, b = 1.0;
    for (int k = 1; k <= q; ++k) {
        double na = a + k + 2, nb = a + b;
        a = na;
        b = nb;
    }
    return b;
}
static double sing_dz2(int q) {
    double a = 0.5, b = 0.0;
    for (int k = 1; k <= q; ++k) {
        double na = a + 0.5 * (k + 1), nb = a + b;
        a = na;
        b = nb;
    }
    return b;
}

static void dubiner_eval(int dof, double z1, double z2, double& phi, double& d1, double& d2) {
    int p, q;
    mode_pq(dof, p, q);
    const double n1 = 2 * (1 + z1) / (1 - z2) - 1;
    const double n2 = z2;
    const double s = (1 - n2) / 2;
    const double sp = std::pow(s, p);
    const double Pp = jacobi(p, 0, 0, n1), Pq = jacobi(q, 2 * p + 1, 0, n2);
    const double dPp = djacobi(p, 0, 0, n1), dPq = djacobi(q, 2 * p + 1, 0, n2);
    phi = Pp * sp * Pq;
    d1 = (2.0 / (1.0 - n2)) * dPp * sp * Pq;
    d2 = ((1 + n1) / (1.0 - n2)) * dPp * sp * Pq + Pp * (sp * dPq - (p / 2.0) * std::pow(s, p - 1) * Pq);
    if (std::isnan(n1)) {
        phi = (p == 0) ? q + 1.0 : 0.0;
        d1 = (p == 1) ? sing_dz1(q) : 0.0;
        d2 = (p == 0) ? 3 * sing_dz2(q) : (p == 1 ? sing_dz2(q + 1) : 0.0);
    }
}

// sort with a strict total order: the parallel sort (OpenMP builds) gives the sequential result
template <typename It, typename Cmp>
static void total_sort(It b, It e, Cmp cmp) {
#ifdef _OPENMP
    __gnu_parallel::sort(b, e, cmp);
#else
    std::sort(b, e, cmp);
#endif
}

static void face_to_master(int f, double z, double& z1, double& z2) {
    // master_triangle.tpp:89-122
    if (f == 0) {
        z1 = -z;
        z2 = z;
    } else if (f == 1) {
        z1 = -1.0;
        z2 = -z;
    } else {
        z1 = z;
        z2 = -1.0;
    }
}

void eval_basis(int p, const double* z1, const double* z2, int n, double* phi) {
    const int nd = (p + 1) * (p + 2) / 2;
    for (int k = 0; k < nd; ++k)
        for (int i = 0; i < n; ++i) {
            double d1, d2;
            dubiner_eval(k, z1[i], z2[i], phi[k * n + i], d1, d2);
        }
}

int build_tables(int p, Tables& t, std::string& err) {
    if (p < 1 || p > 2) {
        err = "polynomial_order must be 1 or 2";
        return DGSW_ERR_UNSUPPORTED;
    }
    std::memset(&t, 0, sizeof(Tables));
    t.p = p;
    t.nd = (p + 1) * (p + 2) / 2;
    Rule2D r = triangle_rule(2 * p);
    Rule1D gl = gauss_legendre_degree(2 * p + 1);
    t.nq = (int)r.w.size();
    t.ng = (int)gl.w.size();
    if (t.nq > MAX_NQ || t.ng > MAX_NG) {
        err = "quadrature larger than the compiled tables";
        return DGSW_ERR_UNSUPPORTED;
    }
    for (int gp = 0; gp < t.nq; ++gp) {
        t.w[gp] = r.w[gp];
        t.psi[0][gp] = -(r.z1[gp] + r.z2[gp]) / 2;
        t.psi[1][gp] = (1 + r.z1[gp]) / 2;
        t.psi[2][gp] = (1 + r.z2[gp]) / 2;
        for (int k = 0; k < t.nd; ++k) {
            double ph, d1, d2;
            dubiner_eval(k, r.z1[gp], r.z2[gp], ph, d1, d2);
            t.phi[k * t.nq + gp] = ph;
            t.dphi[0][k * t.nq + gp] = d1;
            t.dphi[1][k * t.nq + gp] = d2;
            t.mz[0][gp * t.nd + k] = d1 * r.w[gp];
            t.mz[1][gp * t.nd + k] = d2 * r.w[gp];
            t.phiw[gp * t.nd + k] = ph * r.w[gp];
        }
    }
    for (int g = 0; g < t.ng; ++g) t.gw[g] = gl.w[g];
    for (int f = 0; f < 3; ++f)
        for (int g = 0; g < t.ng; ++g) {
            double z1, z2;
            face_to_master(f, gl.z[g], z1, z2);
            t.fpsi[f][0][g] = -(z1 + z2) / 2;
            t.fpsi[f][1][g] = (1 + z1) / 2;
            t.fpsi[f][2][g] = (1 + z2) / 2;
            for (int k = 0; k < t.nd; ++k) {
                double ph, d1, d2;
                dubiner_eval(k, z1, z2, ph, d1, d2);
                t.fphi[f][k * t.ng + g] = ph;
            }
        }
    for (int k = 0; k < t.nd; ++k) {
        int pp, qq;
        mode_pq(k, pp, qq);
        t.minv[k] = (2 * pp + 1) * (pp + qq + 1) / 2.0;  // diagonal of the inverse master mass matrix
    }
    return DGSW_OK;
}

// ------------------------------------------------------------------------------------------------
// Topology. Same results as MeshMetaData (mesh_metadata.cpp:3-85): faces are matched by their
// unordered node pair; here by sorting the 3*ne face keys instead of a hash dictionary. Boundary
// faces take the type of the first boundary chain that contains the node pair as neighbours of the
// first occurrence of the face's first node (AdcircFormat::has_edge semantics).
// ------------------------------------------------------------------------------------------------
int build_topology(const dgsw_mesh* m, Topology& T, std::string& err) {
    const int64_t ne = m->n_elems;
    if (ne <= 0 || m->n_nodes <= 0 || !m->node_xyz || !m->elem_nodes) {
        err = "empty mesh";
        return DGSW_ERR_INVALID_ARGUMENT;
    }
    if (ne > (int64_t)std::numeric_limits<int32_t>::max() / 4) {
        err = "too many elements";
        return DGSW_ERR_UNSUPPORTED;
    }
    T.ne = ne;
    T.nn = m->n_nodes;
    bigvec<std::pair<uint32_t, int32_t>> ord(ne);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < ne; ++i) ord[i] = {m->elem_ids ? m->elem_ids[i] : (uint32_t)i, (int32_t)i};
    if (!std::is_sorted(ord.begin(), ord.end())) total_sort(ord.begin(), ord.end(), std::less<std::pair<uint32_t, int32_t>>());
    T.ids.resize(ne);
    T.src.resize(ne);
    T.enodes.resize(3 * ne);
    // checked in parallel; the first failing element (in ID order) is reported, as a serial scan would
    int64_t bad_dup = ne, bad_node = ne, bad_ccw = ne;
#pragma omp parallel for schedule(static) reduction(min : bad_dup, bad_node, bad_ccw)
    for (int64_t r = 0; r < ne; ++r) {
        if (r > 0 && ord[r].first == ord[r - 1].first) bad_dup = std::min(bad_dup, r);
        T.ids[r] = ord[r].first;
        T.src[r] = ord[r].second;
        bool ok = true;
        for (int v = 0; v < 3; ++v) {
            int32_t n = m->elem_nodes[3 * (int64_t)ord[r].second + v];
            if (n < 0 || n >= m->n_nodes) {
                ok = false;
                n = 0;
            }
            T.enodes[3 * r + v] = n;
        }
        if (!ok) {
            bad_node = std::min(bad_node, r);
            continue;
        }
        const double* X = m->node_xyz;
        const int32_t* nd = &T.enodes[3 * r];
        double det = (X[3 * nd[1]] - X[3 * nd[0]]) * (X[3 * nd[2] + 1] - X[3 * nd[0] + 1]) -
                     (X[3 * nd[1] + 1] - X[3 * nd[0] + 1]) * (X[3 * nd[2]] - X[3 * nd[0]]);
        if (!(det > 0)) bad_ccw = std::min(bad_ccw, r);
    }
    const int64_t first_bad = std::min(bad_dup, std::min(bad_node, bad_ccw));
    if (first_bad < ne) {
        if (first_bad == bad_dup) {
            err = "Fatal Error: duplicate element ID " + std::to_string(ord[first_bad].first);
            return DGSW_ERR_MESH;
        }
        if (first_bad == bad_node) {
            err = "Fatal Error: element node index out of range";
            return DGSW_ERR_MESH;
        }
        err = "element " + std::to_string(T.ids[first_bad]) +
              " is not counter-clockwise (or degenerate); reorder its nodes (the reference swaps coordinates "
              "but not node IDs for such elements, which this library does not reproduce)";
        return DGSW_ERR_UNSUPPORTED;
    }
    // face keys
    struct FK {
        uint64_t key;
        int32_t r;
        int8_t f;
    };
    bigvec<FK> fk(3 * ne);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < ne; ++r)
        for (int f = 0; f < 3; ++f) {
            uint32_t a = (uint32_t)T.enodes[3 * r + (f + 1) % 3], b = (uint32_t)T.enodes[3 * r + (f + 2) % 3];
            fk[3 * r + f] = {(uint64_t)std::min(a, b) << 32 | std::max(a, b), (int32_t)r, (int8_t)f};
        }
    total_sort(fk.begin(), fk.end(), [](const FK& x, const FK& y) {
        return x.key != y.key ? x.key < y.key : (x.r != y.r ? x.r < y.r : x.f < y.f);
    });
    T.nbr.assign(3 * ne, -1);
    T.nbr_face.assign(3 * ne, -1);
    T.btype.assign(3 * ne, 255);
    // boundary chain lookup (AdcircFormat::get_ibtype, adcirc_format.cpp:214-259): the first chain, in
    // the given order, in which the face's two nodes are consecutive (has_edge looks at every occurrence
    // of the first node); a levee chain holds its front and back node strings, searched separately
    // (:230-234); faces joining the two strings at a barrier end are land (is_levee_end, :338-352)
    auto ukey = [](int32_t a, int32_t b) -> uint64_t {
        return (uint64_t)(uint32_t)std::min(a, b) << 32 | (uint32_t)std::max(a, b);
    };
    std::unordered_map<uint64_t, int32_t> edge_seg;   // node pair -> first chain holding it
    std::unordered_map<uint64_t, uint64_t> mirror;    // levee node pair -> node pair across the barrier
    std::unordered_map<uint64_t, int> levee_end;
    for (int32_t s = 0; s < m->n_segments; ++s) {
        const int64_t b = m->seg_offsets[s], e = m->seg_offsets[s + 1];
        for (int64_t i = b; i < e; ++i)
            if (m->seg_nodes[i] < 0 || m->seg_nodes[i] >= m->n_nodes) {
                err = "Fatal Error: boundary node index out of range";
                return DGSW_ERR_MESH;
            }
        if (m->seg_type[s] == DGSW_BC_LEVEE) {
            const int64_t n = (e - b) / 2;
            if ((e - b) % 2 != 0 || n < 2) {
                err = "levee chain " + std::to_string(s) + " must hold n >= 2 front nodes followed by n back nodes";
                return DGSW_ERR_INVALID_ARGUMENT;
            }
            const int32_t* fr = m->seg_nodes + b;
            const int32_t* bk = m->seg_nodes + b + n;
            for (int64_t i = 0; i + 1 < n; ++i) edge_seg.emplace(ukey(fr[i], fr[i + 1]), s);
            for (int64_t i = 0; i + 1 < n; ++i) edge_seg.emplace(ukey(bk[i], bk[i + 1]), s);
            // AdcircFormat::get_internal_node_pair (:261-318): front pair <-> back pair
            for (int64_t i = 0; i + 1 < n; ++i) mirror.emplace(ukey(fr[i], fr[i + 1]), ukey(bk[i], bk[i + 1]));
            for (int64_t i = 0; i + 1 < n; ++i) mirror.emplace(ukey(bk[i], bk[i + 1]), ukey(fr[i], fr[i + 1]));
            levee_end.emplace(ukey(fr[0], bk[0]), 1);
            levee_end.emplace(ukey(fr[n - 1], bk[n - 1]), 1);
        } else {
            for (int64_t i = b; i + 1 < e; ++i) edge_seg.emplace(ukey(m->seg_nodes[i], m->seg_nodes[i + 1]), s);
        }
    }
    auto lookup_type = [&](int32_t n0, int32_t n1) -> int {
        auto it = edge_seg.find(ukey(n0, n1));
        if (it != edge_seg.end()) return m->seg_type[it->second];
        if (levee_end.count(ukey(n0, n1))) return DGSW_BC_LAND;
        return -1;
    };
    // levee faces: the element across the barrier (first element holding the mirrored edge)
    std::vector<int32_t> lev_nbr(3 * ne, -1);
    auto first_holder = [&](uint64_t key) -> int32_t {
        auto it = std::lower_bound(fk.begin(), fk.end(), key, [](const FK& x, uint64_t k) { return x.key < k; });
        return (it != fk.end() && it->key == key) ? it->r : -1;
    };
    for (size_t i = 0; i < fk.size();) {
        size_t j = i + 1;
        while (j < fk.size() && fk[j].key == fk[i].key) ++j;
        if (j - i > 2) {
            err = "Fatal Error: edge shared by more than two elements";
            return DGSW_ERR_MESH;
        }
        if (j - i == 2) {
            const FK& A = fk[i];
            const FK& B = fk[i + 1];
            if (A.r == B.r) {
                err = "Fatal Error: degenerate element";
                return DGSW_ERR_MESH;
            }
            T.nbr[3 * A.r + A.f] = B.r;
            T.nbr_face[3 * A.r + A.f] = B.f;
            T.btype[3 * A.r + A.f] = DGSW_BC_INTERNAL;
            T.nbr[3 * B.r + B.f] = A.r;
            T.nbr_face[3 * B.r + B.f] = A.f;
            T.btype[3 * B.r + B.f] = DGSW_BC_INTERNAL;
        } else {
            const FK& A = fk[i];
            int32_t n0 = T.enodes[3 * A.r + (A.f + 1) % 3], n1 = T.enodes[3 * A.r + (A.f + 2) % 3];
            int bt = lookup_type(n0, n1);
            if (bt < 0) {
                err = "Fatal Error: boundary not found, unable to assign BOUNDARY_TYPE to given node_pair (" +
                      std::to_string(n0) + ", " + std::to_string(n1) + ")!";
                return DGSW_ERR_MESH;
            }
            if (bt != DGSW_BC_LAND && bt != DGSW_BC_TIDE && bt != DGSW_BC_FLOW && bt != DGSW_BC_FUNCTION &&
                bt != DGSW_BC_OUTFLOW && bt != DGSW_BC_LEVEE) {
                err = "unsupported boundary type " + std::to_string(bt);
                return DGSW_ERR_UNSUPPORTED;
            }
            T.btype[3 * A.r + A.f] = (uint8_t)bt;
            if (bt == DGSW_BC_LEVEE) {
                const int32_t across = first_holder(mirror.at(ukey(n0, n1)));
                if (across < 0) {
                    err = "Fatal Error: no element across the barrier from node pair (" + std::to_string(n0) + ", " +
                          std::to_string(n1) + ")";
                    return DGSW_ERR_MESH;
                }
                lev_nbr[3 * A.r + A.f] = across;
            }
        }
        i = j;
    }
    // levee interfaces pair the raw boundaries keyed (element, element across) with their mirror image
    // (swe_pre_create_intface.hpp:38-78); a key seen twice keeps its first face, as std::map::emplace does
    for (int64_t r = 0; r < ne; ++r)
        for (int f = 0; f < 3; ++f) {
            const int32_t b = lev_nbr[3 * r + f];
            if (b < 0) continue;
            bool first = true;
            for (int g = 0; g < f; ++g) first = first && lev_nbr[3 * r + g] != b;
            int fb = -1;
            for (int g = 0; g < 3 && fb < 0; ++g)
                if (lev_nbr[3 * (int64_t)b + g] == (int32_t)r) fb = g;
            if (first && fb >= 0) {
                T.nbr[3 * r + f] = b;
                T.nbr_face[3 * r + f] = (int8_t)fb;
            }
        }
    // two faces of one element against the same neighbour would collide in the reference's
    // (element, neighbour) keyed maps; reject such meshes
    for (int64_t r = 0; r < ne; ++r)
        for (int f = 0; f < 3; ++f)
            for (int g = f + 1; g < 3; ++g)
                if (T.nbr[3 * r + f] >= 0 && T.nbr[3 * r + f] == T.nbr[3 * r + g] &&
                    T.btype[3 * r + f] == T.btype[3 * r + g]) {
                    err = "Fatal Error: two elements share more than one edge";
                    return DGSW_ERR_MESH;
                }
    // interfaces in (in, ex) order, in = smaller reference ID (swe_pre_create_intface.hpp:14-34): the
    // internal ones, then the levee ones (ProblemInterfaceTypes order)
    T.intf.clear();
    std::vector<int32_t> intf_of_face(3 * ne, -1);
    {
        // counts per element, prefix sums, then each element writes its own interfaces in place
        std::vector<int32_t> cnt(2 * ne + 1, 0);
        const int kinds[2] = {DGSW_BC_INTERNAL, DGSW_BC_LEVEE};
#pragma omp parallel for schedule(static)
        for (int64_t r = 0; r < ne; ++r)
            for (int k = 0; k < 2; ++k) {
                int n = 0;
                for (int f = 0; f < 3; ++f) n += (T.nbr[3 * r + f] > r && T.btype[3 * r + f] == kinds[k]) ? 1 : 0;
                cnt[k * ne + r + 1] = n;
            }
        for (int64_t i = 0; i < 2 * ne; ++i) cnt[i + 1] += cnt[i];
        T.n_intf_internal = cnt[ne];
        T.intf.resize((size_t)4 * cnt[2 * ne]);
        for (int k = 0; k < 2; ++k) {
#pragma omp parallel for schedule(static)
            for (int64_t r = 0; r < ne; ++r) {
                // faces of r with a larger neighbour, ordered by the neighbour
                int fs[3], n = 0;
                for (int f = 0; f < 3; ++f)
                    if (T.nbr[3 * r + f] > r && T.btype[3 * r + f] == kinds[k]) fs[n++] = f;
                std::sort(fs, fs + n, [&](int a, int b) { return T.nbr[3 * r + a] < T.nbr[3 * r + b]; });
                int32_t idx = cnt[k * ne + r];
                for (int j = 0; j < n; ++j, ++idx) {
                    const int f = fs[j];
                    const int32_t e = T.nbr[3 * r + f];
                    const int fe = T.nbr_face[3 * r + f];
                    T.intf[4 * (size_t)idx] = (int32_t)r;
                    T.intf[4 * (size_t)idx + 1] = e;
                    T.intf[4 * (size_t)idx + 2] = f;
                    T.intf[4 * (size_t)idx + 3] = fe;
                    intf_of_face[3 * r + f] = idx;
                    intf_of_face[3 * (int64_t)e + fe] = idx;
                }
            }
        }
    }
    // boundaries grouped by type (Land, Tide, Flow, Function tuple order), each by (element, face)
    T.bnd.clear();
    std::vector<int64_t> bnd_of_face(3 * ne, -1);
    for (int bt : {DGSW_BC_LAND, DGSW_BC_TIDE, DGSW_BC_FLOW, DGSW_BC_FUNCTION}) {
        for (int64_t r = 0; r < ne; ++r)
            for (int f = 0; f < 3; ++f)
                if (T.btype[3 * r + f] == bt) {
                    bnd_of_face[3 * r + f] = (int64_t)T.bnd.size() / 3;
                    T.bnd.push_back((int32_t)r);
                    T.bnd.push_back(f);
                    T.bnd.push_back(bt);
                }
    }
    // per element accumulation order: its interfaces by creation index, then its boundaries
    T.order_count.assign(ne, 0);
    T.order_face.assign(3 * ne, 0);
    T.is_in.assign(3 * ne, 0);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < ne; ++r) {
        std::pair<int64_t, int> items[3];
        int n = 0;
        for (int f = 0; f < 3; ++f)
            if (intf_of_face[3 * r + f] >= 0) items[n++] = {intf_of_face[3 * r + f], f};
        std::sort(items, items + n);
        int ni = n;
        for (int f = 0; f < 3; ++f)
            if (bnd_of_face[3 * r + f] >= 0) items[n++] = {bnd_of_face[3 * r + f], f};
        std::sort(items + ni, items + n);
        T.order_count[r] = (uint8_t)n;
        for (int k = 0; k < n; ++k) T.order_face[3 * r + k] = (uint8_t)items[k].second;
        // the element owns the flux evaluation of its boundary faces and of interfaces to larger IDs
        for (int f = 0; f < 3; ++f) T.is_in[3 * r + f] = (T.nbr[3 * r + f] > r || T.nbr[3 * r + f] < 0) ? 1 : 0;
    }
    return DGSW_OK;
}

// ------------------------------------------------------------------------------------------------
// Device order and tiles: Morton order of element centroids, cut into tiles of `tile` elements.
// Each tile lists the edges its elements need: interior edges once per tile (an edge between two
// tiles appears in both lists and is evaluated by both CTAs with the same code), boundary edges
// with a boundary object (land, tide, flow, function). Outflow faces have no object and contribute nothing.
// ------------------------------------------------------------------------------------------------
static uint64_t spread21(uint64_t v) {
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
}

void element_geometry(const double* X, const int32_t* nd, double out[5]) {
    const double J00 = (X[3 * nd[1]] - X[3 * nd[0]]) / 2.0, J01 = (X[3 * nd[2]] - X[3 * nd[0]]) / 2.0;
    const double J10 = (X[3 * nd[1] + 1] - X[3 * nd[0] + 1]) / 2.0, J11 = (X[3 * nd[2] + 1] - X[3 * nd[0] + 1]) / 2.0;
    const double det = J00 * J11 - J10 * J01;
    const double invdet = 1.0 / det;  // 2x2 cofactor inverse
    out[0] = J11 * invdet;
    out[1] = -J01 * invdet;
    out[2] = -J10 * invdet;
    out[3] = J00 * invdet;
    out[4] = std::abs(det);
}

void face_geometry(const double* X, const int32_t* nd, int f, double& nx, double& ny, double& sJ) {
    const int a = nd[(f + 1) % 3], b = nd[(f + 2) % 3];
    const double dx = X[3 * b] - X[3 * a], dy = X[3 * b + 1] - X[3 * a + 1];
    double J00 = (X[3 * nd[1]] - X[3 * nd[0]]) / 2.0, J01 = (X[3 * nd[2]] - X[3 * nd[0]]) / 2.0;
    double J10 = (X[3 * nd[1] + 1] - X[3 * nd[0] + 1]) / 2.0, J11 = (X[3 * nd[2] + 1] - X[3 * nd[0] + 1]) / 2.0;
    const double det = J00 * J11 - J10 * J01;
    const double cw = det / std::abs(det);
    const double length = std::hypot(dx, dy);
    nx = cw * dy / length;
    ny = -cw * dx / length;
    sJ = std::sqrt(std::pow(dx, 2.0) + std::pow(dy, 2.0)) / 2.0;
}

// open-addressing map from non-negative keys to small ints, for the per-tile edge and halo lookups (a few
// hundred entries per tile); clear() forgets only the slots in use
struct FlatMap {
    static constexpr int CAP = 4096;  // > 2 x the largest tile list (1022 edges, 3 x 256 + halo faces)
    std::vector<int64_t> keys = std::vector<int64_t>(CAP, -1);
    std::vector<int32_t> vals = std::vector<int32_t>(CAP, 0);
    std::vector<int32_t> used;
    static uint32_t slot(int64_t k) { return (uint32_t)(((uint64_t)k * 0x9E3779B97F4A7C15ull) >> 52) & (CAP - 1); }
    int find(int64_t k) const {
        for (uint32_t i = slot(k);; i = (i + 1) & (CAP - 1)) {
            if (keys[i] == k) return vals[i];
            if (keys[i] < 0) return -1;
        }
    }
    void insert(int64_t k, int32_t v) {
        uint32_t i = slot(k);
        while (keys[i] >= 0) i = (i + 1) & (CAP - 1);
        keys[i] = k;
        vals[i] = v;
        used.push_back((int32_t)i);
    }
    int size() const { return (int)used.size(); }
    void clear() {
        for (int32_t i : used) keys[i] = -1;
        used.clear();
    }
};

int build_tiling(const Topology& T, const double* X, int tile, bool morton, Tiling& out, std::string& err) {
    const int64_t ne = T.ne;
    if (tile != 64 && tile != 128 && tile != 256) {
        err = "tile must be 64, 128 or 256";
        return DGSW_ERR_INVALID_ARGUMENT;
    }
    out.tile = tile;
    out.ref_of_dev.resize(ne);
    std::iota(out.ref_of_dev.begin(), out.ref_of_dev.end(), 0);
    if (morton) {
        // Morton order of centroids within each ensemble member (members overlap in space), members
        // kept in their order so that tiles rarely straddle two members
        const bool grouped = !T.group.empty();
        int32_t ng = 1;
        if (grouped)
            for (int64_t r = 0; r < ne; ++r) ng = std::max(ng, T.group[r] + 1);
        std::vector<double> xmin(ng, 1e300), xmax(ng, -1e300), ymin(ng, 1e300), ymax(ng, -1e300);
        std::vector<double> cx(ne), cy(ne);
        for (int64_t r = 0; r < ne; ++r) {
            const int32_t* nd = &T.enodes[3 * r];
            const int32_t gi = grouped ? T.group[r] : 0;
            cx[r] = (X[3 * nd[0]] + X[3 * nd[1]] + X[3 * nd[2]]) / 3.0;
            cy[r] = (X[3 * nd[0] + 1] + X[3 * nd[1] + 1] + X[3 * nd[2] + 1]) / 3.0;
            xmin[gi] = std::min(xmin[gi], cx[r]);
            xmax[gi] = std::max(xmax[gi], cx[r]);
            ymin[gi] = std::min(ymin[gi], cy[r]);
            ymax[gi] = std::max(ymax[gi], cy[r]);
        }
        std::vector<uint64_t> key(ne);
#pragma omp parallel for schedule(static)
        for (int64_t r = 0; r < ne; ++r) {
            const int32_t gi = grouped ? T.group[r] : 0;
            double span = std::max(xmax[gi] - xmin[gi], ymax[gi] - ymin[gi]);
            if (span <= 0) span = 1;
            uint64_t ix = (uint64_t)std::min(2097151.0, std::floor((cx[r] - xmin[gi]) / span * 2097151.0));
            uint64_t iy = (uint64_t)std::min(2097151.0, std::floor((cy[r] - ymin[gi]) / span * 2097151.0));
            key[r] = spread21(ix) | spread21(iy) << 1;
        }
        // (member, Morton key, element): the stable order of (member, key)
        total_sort(out.ref_of_dev.begin(), out.ref_of_dev.end(), [&](int32_t a, int32_t b) {
            const int32_t ga = grouped ? T.group[a] : 0, gb = grouped ? T.group[b] : 0;
            return ga != gb ? ga < gb : (key[a] != key[b] ? key[a] < key[b] : a < b);
        });
    }
    out.dev_of_ref.resize(ne);
    for (int64_t d = 0; d < ne; ++d) out.dev_of_ref[out.ref_of_dev[d]] = (int32_t)d;
    out.ntiles = (ne + tile - 1) / tile;
    out.tile_edge_off.assign(out.ntiles + 1, 0);
    out.tile_halo_off.assign(out.ntiles + 1, 0);
    out.edges.clear();
    out.egeo.clear();
    out.halo.clear();
    out.eslot.assign(2 * ne, 0);
    out.max_edges = 0;
    out.max_halo = 0;
    std::vector<int32_t> iface(3 * ne, -1);
    const int64_t n_intf = (int64_t)T.intf.size() / 4;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n_intf; ++i) {
        iface[3 * (int64_t)T.intf[4 * i] + T.intf[4 * i + 2]] = (int32_t)i;
        iface[3 * (int64_t)T.intf[4 * i + 1] + T.intf[4 * i + 3]] = (int32_t)i;
    }
    std::vector<int32_t> bface(3 * ne, -1);
    for (size_t i = 0; i < T.bnd.size() / 3; ++i) bface[3 * (int64_t)T.bnd[3 * i] + T.bnd[3 * i + 1]] = (int32_t)i;
    // tiles are independent: each builds its own edge, geometry and halo lists (in parallel), and the
    // lists are concatenated in tile order
    struct TileLists {
        std::vector<int32_t> te;  // edge records
        std::vector<double> tg;   // edge geometry
        std::vector<int32_t> halo;
    };
    std::vector<TileLists> lists((size_t)out.ntiles);
    int overflow = 0;
#pragma omp parallel
    {
        FlatMap local_edge, local_halo;
#pragma omp for schedule(dynamic, 16) reduction(| : overflow)
        for (int64_t t = 0; t < out.ntiles; ++t) {
            local_edge.clear();
            local_halo.clear();
            std::vector<int32_t>& te = lists[t].te;
            te.reserve(4 * (size_t)(3 * tile / 2 + 32));
            std::vector<double>& tg = lists[t].tg;
            std::vector<int32_t>& halo = lists[t].halo;
            const int64_t d0 = t * tile, d1 = std::min(ne, d0 + tile);
            // trace slot of (element in reference order, face)
            auto trace_slot = [&](int32_t r, int f) -> int32_t {
                const int64_t d = out.dev_of_ref[r];
                if (d >= d0 && d < d1) return (int32_t)(3 * (d - d0) + f);
                const int64_t key = 3 * (int64_t)r + f;
                const int found = local_halo.find(key);
                if (found >= 0) return 3 * tile + found;
                const int h = local_halo.size();
                local_halo.insert(key, h);
                halo.push_back((int32_t)d);
                halo.push_back(f);
                return 3 * tile + h;
            };
            for (int64_t d = d0; d < d1; ++d) {
                const int32_t r = out.ref_of_dev[d];
                uint32_t slots[3] = {1023, 1023, 1023};
                for (int f = 0; f < 3; ++f) {
                    const int64_t ii = iface[3 * (int64_t)r + f];
                    const int64_t bi = bface[3 * (int64_t)r + f];
                    if (ii >= 0) {
                        const int found = local_edge.find(ii);
                        if (found >= 0) {
                            slots[f] = (uint32_t)found;
                            continue;
                        }
                        const int idx = (int)(te.size() / 4);
                        local_edge.insert(ii, idx);
                        slots[f] = (uint32_t)idx;
                        const int32_t in = T.intf[4 * ii], ex = T.intf[4 * ii + 1];
                        const int fin = T.intf[4 * ii + 2], fex = T.intf[4 * ii + 3];
                        te.push_back(trace_slot(in, fin));
                        te.push_back(trace_slot(ex, fex));
                        // levee interfaces carry their index among the levee interfaces above bit 8
                        const bool lev = ii >= T.n_intf_internal;
                        te.push_back(lev ? (fin | fex << 2 | EK_LEVEE << 4 | (int32_t)(ii - T.n_intf_internal) << 8)
                                         : (fin | fex << 2 | EK_INTERIOR << 4));
                        te.push_back(out.dev_of_ref[in]);
                        double nx, ny, sJ;
                        face_geometry(X, &T.enodes[3 * (int64_t)in], fin, nx, ny, sJ);
                        tg.push_back(nx);
                        tg.push_back(ny);
                        tg.push_back(sJ);
                    } else if (bi >= 0) {
                        const int idx = (int)(te.size() / 4);
                        slots[f] = (uint32_t)idx;
                        const int bt = T.bnd[3 * bi + 2];
                        const int kind = bt == DGSW_BC_LAND   ? EK_LAND
                                         : bt == DGSW_BC_TIDE ? EK_TIDE
                                         : bt == DGSW_BC_FLOW ? EK_FLOW
                                                              : EK_FUNCTION;
                        // tide / flow faces carry their forcing record as -2 - index in the b slot
                        const int32_t fidx = (kind == EK_TIDE || kind == EK_FLOW) ? T.bnd_force[bi] : -1;
                        te.push_back((int32_t)(3 * (d - d0) + f));
                        te.push_back(fidx >= 0 ? -2 - fidx : -1);
                        te.push_back(f | kind << 4);
                        te.push_back((int32_t)d);
                        double nx, ny, sJ;
                        face_geometry(X, &T.enodes[3 * (int64_t)r], f, nx, ny, sJ);
                        tg.push_back(nx);
                        tg.push_back(ny);
                        tg.push_back(sJ);
                    }
                }
                int32_t roles = 0;
                for (int f = 0; f < 3; ++f) roles |= (T.is_in[3 * r + f] ? 1 : 0) << f;
                int32_t ord = T.order_count[r];
                for (int k = 0; k < T.order_count[r]; ++k) ord |= T.order_face[3 * r + k] << (2 + 2 * k);
                out.eslot[2 * d] = (int32_t)(slots[0] | slots[1] << 10 | slots[2] << 20);
                out.eslot[2 * d + 1] = roles | ord << 3;
            }
            if (te.size() / 4 > 1022) overflow = 1;
        }
    }
    if (overflow) {
        err = "tile edge list overflow";
        return DGSW_ERR_INVALID_ARGUMENT;
    }
    // offsets by a prefix sum over the tiles, then every tile copies its lists into place
    std::vector<int64_t> eo(out.ntiles + 1, 0), ho(out.ntiles + 1, 0);
    for (int64_t t = 0; t < out.ntiles; ++t) {
        eo[t + 1] = eo[t] + (int64_t)lists[t].te.size() / 4;
        ho[t + 1] = ho[t] + (int64_t)lists[t].halo.size() / 2;
        out.max_edges = std::max(out.max_edges, (int)(lists[t].te.size() / 4));
        out.max_halo = std::max(out.max_halo, (int)(lists[t].halo.size() / 2));
    }
    if (eo[out.ntiles] >= std::numeric_limits<int32_t>::max() || ho[out.ntiles] >= std::numeric_limits<int32_t>::max()) {
        err = "too many tile edges";
        return DGSW_ERR_UNSUPPORTED;
    }
    out.edges.resize((size_t)4 * eo[out.ntiles]);
    out.egeo.resize((size_t)3 * eo[out.ntiles]);
    out.halo.resize((size_t)2 * ho[out.ntiles]);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t t = 0; t < out.ntiles; ++t) {
        TileLists& L = lists[t];
        out.tile_edge_off[t] = (int32_t)eo[t];
        out.tile_halo_off[t] = (int32_t)ho[t];
        std::copy(L.te.begin(), L.te.end(), out.edges.begin() + 4 * eo[t]);
        std::copy(L.tg.begin(), L.tg.end(), out.egeo.begin() + 3 * eo[t]);
        std::copy(L.halo.begin(), L.halo.end(), out.halo.begin() + 2 * ho[t]);
        std::vector<int32_t>().swap(L.te);
        std::vector<double>().swap(L.tg);
        std::vector<int32_t>().swap(L.halo);
    }
    out.tile_edge_off[out.ntiles] = (int32_t)((int64_t)out.edges.size() / 4);
    out.tile_halo_off[out.ntiles] = (int32_t)((int64_t)out.halo.size() / 2);
    return DGSW_OK;
}

// ------------------------------------------------------------------------------------------------
// Tide / flow forcing and Manning friction data
// ------------------------------------------------------------------------------------------------
int build_forcing(const dgsw_mesh* m, Topology& T, int p, Forcing& out, std::string& err) {
    const size_t nb = T.bnd.size() / 3;
    T.bnd_force.assign(nb, -1);
    out.face.clear();
    out.con.clear();
    bool forced = false;
    for (size_t i = 0; i < nb; ++i) forced = forced || T.bnd[3 * i + 2] == DGSW_BC_TIDE || T.bnd[3 * i + 2] == DGSW_BC_FLOW;
    if (!forced) return DGSW_OK;
    if (m->n_forcing < 0 || (m->n_forcing > 0 && !m->forcing)) {
        err = "invalid forcing block list";
        return DGSW_ERR_INVALID_ARGUMENT;
    }
    // node -> position in each block; the reference keeps one map per block keyed by node ID
    std::vector<std::unordered_map<int32_t, int32_t>> pos(m->n_forcing);
    for (int32_t b = 0; b < m->n_forcing; ++b) {
        const dgsw_forcing_block& B = m->forcing[b];
        if ((B.type != DGSW_BC_TIDE && B.type != DGSW_BC_FLOW) || B.n_nodes < 0 || B.n_constituents < 0 ||
            (B.n_nodes > 0 && !B.nodes) ||
            (B.n_constituents > 0 && (!B.frequency || !B.forcing_fact || !B.equilib_arg)) ||
            ((int64_t)B.n_nodes * B.n_constituents > 0 && (!B.amplitude || !B.phase))) {
            err = "forcing block " + std::to_string(b) + " is malformed";
            return DGSW_ERR_INVALID_ARGUMENT;
        }
        for (int32_t j = 0; j < B.n_nodes; ++j) {
            const int32_t n = B.nodes[j];
            if (n < 0 || n >= m->n_nodes) {
                err = "forcing block " + std::to_string(b) + ": node index out of range";
                return DGSW_ERR_MESH;
            }
            // the reference appends a repeated node's values to the same per-node lists, which shifts
            // its constituents; such input is rejected here instead
            if (!pos[b].emplace(n, j).second) {
                err = "forcing block " + std::to_string(b) + " lists node " + std::to_string(n) + " twice";
                return DGSW_ERR_MESH;
            }
        }
    }
    const Rule1D gl = gauss_legendre_degree(2 * p + 1);
    const int ng = (int)gl.z.size();
    for (size_t i = 0; i < nb; ++i) {
        const int bt = T.bnd[3 * i + 2];
        if (bt != DGSW_BC_TIDE && bt != DGSW_BC_FLOW) continue;
        const int64_t r = T.bnd[3 * i];
        const int f = T.bnd[3 * i + 1];
        // Shape::GetBoundaryNodeID: the face's nodes (f+1)%3, (f+2)%3
        const int32_t n0 = T.enodes[3 * r + (f + 1) % 3], n1 = T.enodes[3 * r + (f + 2) % 3];
        int32_t blk = -1, p0 = 0, p1 = 0;
        for (int32_t b = 0; b < m->n_forcing && blk < 0; ++b) {
            if (m->forcing[b].type != bt) continue;
            auto a = pos[b].find(n0), c = pos[b].find(n1);
            if (a != pos[b].end() && c != pos[b].end()) {
                blk = b;
                p0 = a->second;
                p1 = c->second;
            }
        }
        if (blk < 0) {
            err = bt == DGSW_BC_TIDE ? "Fatal Error: unable to find tide data!" : "Fatal Error: unable to find flow data!";
            return DGSW_ERR_MESH;
        }
        const dgsw_forcing_block& B = m->forcing[blk];
        T.bnd_force[i] = (int32_t)(out.face.size() / 2);
        out.face.push_back((int32_t)(out.con.size() / FORCE_STRIDE));
        out.face.push_back(B.n_constituents);
        for (int32_t c = 0; c < B.n_constituents; ++c) {
            double rec[FORCE_STRIDE] = {0};
            rec[0] = B.frequency[c];
            rec[1] = B.forcing_fact[c];
            rec[2] = B.equilib_arg[c];
            const size_t row = (size_t)c * B.n_nodes;
            // ComputeBoundaryNodalUgp: nodal values times the boundary shape functions (1 - z)/2, (1 + z)/2
            for (int g = 0; g < ng; ++g) {
                const double N1 = (1.0 - gl.z[g]) / 2.0, N2 = (1.0 + gl.z[g]) / 2.0;
                rec[3 + g] = B.amplitude[row + p0] * N1 + B.amplitude[row + p1] * N2;
                rec[3 + MAX_NG + g] = B.phase[row + p0] * N1 + B.phase[row + p1] * N2;
            }
            out.con.insert(out.con.end(), rec, rec + FORCE_STRIDE);
        }
    }
    return DGSW_OK;
}

int build_levees(const dgsw_mesh* m, const Topology& T, int p, const double* X, const dgsw_config& cfg,
                 std::vector<double>& out, std::string& err) {
    out.clear();
    const int64_t n_lev = (int64_t)T.intf.size() / 4 - T.n_intf_internal;
    if (n_lev <= 0) return DGSW_OK;
    if (n_lev >= ((int64_t)1 << 23)) {
        err = "too many levee interfaces";
        return DGSW_ERR_UNSUPPORTED;
    }
    if (m->n_levee_pairs < 0 || (m->n_levee_pairs > 0 && (!m->levee_nodes || !m->levee_data))) {
        err = "invalid levee pair list";
        return DGSW_ERR_INVALID_ARGUMENT;
    }
    // levee_is_data: keyed by the ordered (front, back) pair; a repeated key keeps the last line
    std::map<std::pair<int32_t, int32_t>, int32_t> data;
    for (int32_t k = 0; k < m->n_levee_pairs; ++k) data[{m->levee_nodes[2 * k], m->levee_nodes[2 * k + 1]}] = k;
    const Rule1D gl = gauss_legendre_degree(2 * p + 1);
    const int ng = (int)gl.z.size();
    const double cos_lat0 = std::cos(cfg.sp_lat0_deg * 3.14159265359 / 180.0);  // the reference's PI
    out.assign((size_t)LEVEE_STRIDE * n_lev, 0.0);
    for (int64_t l = 0; l < n_lev; ++l) {
        const int64_t i = T.n_intf_internal + l;
        const int32_t in = T.intf[4 * i], ex = T.intf[4 * i + 1], fin = T.intf[4 * i + 2], fex = T.intf[4 * i + 3];
        const int32_t ni[2] = {T.enodes[3 * (int64_t)in + (fin + 1) % 3], T.enodes[3 * (int64_t)in + (fin + 2) % 3]};
        const int32_t nx_[2] = {T.enodes[3 * (int64_t)ex + (fex + 1) % 3], T.enodes[3 * (int64_t)ex + (fex + 2) % 3]};
        double v[3][2];
        for (int k = 0; k < 2; ++k) {
            auto it = data.find({ni[k], nx_[1 - k]});
            if (it == data.end()) it = data.find({nx_[1 - k], ni[k]});
            if (it == data.end()) {
                err = "Fatal Error: unable to find levee data!";
                return DGSW_ERR_MESH;
            }
            for (int c = 0; c < 3; ++c) v[c][k] = m->levee_data[3 * (int64_t)it->second + c];
        }
        double* o = &out[(size_t)LEVEE_STRIDE * l];
        double nx, ny, sJ;
        face_geometry(X, &T.enodes[3 * (int64_t)in], fin, nx, ny, sJ);
        o[0] = nx;
        o[1] = ny;
        for (int g = 0; g < ng; ++g) {
            // ComputeBoundaryNodalUgpIN: (1 - z)/2, (1 + z)/2 on the in side's face nodes
            const double N1 = (1.0 - gl.z[g]) / 2.0, N2 = (1.0 + gl.z[g]) / 2.0;
            for (int c = 0; c < 3; ++c) o[2 + c * MAX_NG + g] = v[c][0] * N1 + v[c][1] * N2;
        }
        // spherical correction at the in side's Gauss points, for both sides: the ex side's value at its
        // Gauss point ng-1-g is the in side's at g (swe_pre_init_data.hpp:80-101)
        for (int g = 0; g < ng; ++g) {
            double sp = 1.0;
            if (cfg.spherical) {
                const double wa = (1.0 - gl.z[g]) / 2.0, wb = (1.0 + gl.z[g]) / 2.0;
                const double y = X[3 * (int64_t)ni[0] + 1] * wa + X[3 * (int64_t)ni[1] + 1] * wb;
                sp = cos_lat0 / std::cos(y / cfg.sp_R);
            }
            o[2 + 3 * MAX_NG + g] = sp;
            o[2 + 4 * MAX_NG + (ng - 1 - g)] = sp;
        }
    }
    return DGSW_OK;
}

void manning_factor(const Topology& T, const double* node_n, double g, std::vector<double>& out) {
    out.assign(T.ne, 0.0);
    for (int64_t r = 0; r < T.ne; ++r) {
        double s = 0.0;
        for (int v = 0; v < 3; ++v) s += node_n[T.enodes[3 * r + v]];
        out[r] = g * std::pow(s / 3.0, 2);
    }
}

// ------------------------------------------------------------------------------------------------
// FP64 projections (initialize_data_serial, swe_pre_init_data.hpp:9-64) and wet/dry initialisation
// ------------------------------------------------------------------------------------------------
static void elem_geom(const double* X, const int32_t* nd, double& aJ) {
    double J00 = (X[3 * nd[1]] - X[3 * nd[0]]) / 2.0, J01 = (X[3 * nd[2]] - X[3 * nd[0]]) / 2.0;
    double J10 = (X[3 * nd[1] + 1] - X[3 * nd[0] + 1]) / 2.0, J11 = (X[3 * nd[2] + 1] - X[3 * nd[0] + 1]) / 2.0;
    aJ = std::abs(J00 * J11 - J10 * J01);
}

// L2ProjectionNode: ((nodal * psi_gp) * int_phi_fact) * m_inv
static void l2_node(const Tables& tb, double aJ, const double nodal[3], double* out) {
    double a[MAX_NQ];
    for (int gp = 0; gp < tb.nq; ++gp) {
        double s = 0;
        for (int n = 0; n < 3; ++n) s += nodal[n] * tb.psi[n][gp];
        a[gp] = s;
    }
    for (int k = 0; k < tb.nd; ++k) {
        double s = 0;
        for (int gp = 0; gp < tb.nq; ++gp) s += a[gp] * (tb.phiw[gp * tb.nd + k] * aJ);
        out[k] = s * (tb.minv[k] / aJ);
    }
}

void project_bathymetry(const Topology& T, const double* X, const Tables& tb, std::vector<double>& bath) {
    bath.assign(T.ne * tb.nd, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < T.ne; ++r) {
        const int32_t* nd = &T.enodes[3 * r];
        double aJ;
        elem_geom(X, nd, aJ);
        double z[3] = {X[3 * nd[0] + 2], X[3 * nd[1] + 2], X[3 * nd[2] + 2]};
        l2_node(tb, aJ, z, &bath[r * tb.nd]);
    }
}

void project_initial_condition(const Topology& T, const double* X, const Tables& tb, const dgsw_config& cfg,
                               std::vector<double>& q) {
    const int nd = tb.nd;
    q.assign(T.ne * 3 * nd, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < T.ne; ++r) {
        const int32_t* no = &T.enodes[3 * r];
        double aJ;
        elem_geom(X, no, aJ);
        double* qe = &q[r * 3 * nd];
        const double* params = T.group.empty() ? cfg.fn_params : &T.group_params[(size_t)T.group[r] * DGSW_FN_PARAMS];
        if (cfg.ic_type == 0) {
            for (int v = 0; v < 3; ++v) {
                double nodal[3] = {cfg.ic_const[v], cfg.ic_const[v], cfg.ic_const[v]};
                l2_node(tb, aJ, nodal, qe + v * nd);
            }
        } else {
            double fg[3][MAX_NQ];
            for (int gp = 0; gp < tb.nq; ++gp) {
                double x = X[3 * no[0]] * tb.psi[0][gp] + X[3 * no[1]] * tb.psi[1][gp] + X[3 * no[2]] * tb.psi[2][gp];
                double y = X[3 * no[0] + 1] * tb.psi[0][gp] + X[3 * no[1] + 1] * tb.psi[1][gp] +
                           X[3 * no[2] + 1] * tb.psi[2][gp];
                dgsw_fn3 f = dgsw_fn_ic(cfg.function_set, params, 0.0, x, y);
                fg[0][gp] = f.ze;
                fg[1][gp] = f.qx;
                fg[2][gp] = f.qy;
            }
            for (int v = 0; v < 3; ++v)
                for (int k = 0; k < nd; ++k) {
                    double s = 0;
                    for (int gp = 0; gp < tb.nq; ++gp) s += fg[v][gp] * (tb.phiw[gp * nd + k] * aJ);
                    qe[v * nd + k] = s * (tb.minv[k] / aJ);
                }
        }
    }
}

// basis -> vertex values through T_basis_linear (first three modes, basis_dubiner_2D.cpp:213-234)
static inline void to_vertices(const double* qv, double out[3]) {
    out[0] = qv[0] - qv[1] - qv[2];
    out[1] = qv[0] - qv[1] + qv[2];
    out[2] = qv[0] + 2.0 * qv[1];
}
// vertex values -> basis through T_linear_basis (:236-257); higher modes become zero
static inline void from_vertices(const double v[3], double* qv, int nd) {
    qv[0] = v[0] * (1.0 / 3.0) + v[1] * (1.0 / 3.0) + v[2] * (1.0 / 3.0);
    qv[1] = v[0] * (-1.0 / 6.0) + v[1] * (-1.0 / 6.0) + v[2] * (1.0 / 3.0);
    qv[2] = v[0] * (-1.0 / 2.0) + v[1] * (1.0 / 2.0);
    for (int k = 3; k < nd; ++k) qv[k] = 0.0;
}

void init_wet_dry(const Topology& T, const double* X, const Tables& tb, const dgsw_config& cfg, std::vector<double>& q,
                  std::vector<uint8_t>& wet) {
    wet.assign(T.ne, 1);
    if (!cfg.wetting_drying) return;
    const double thr = 1.0e6 * cfg.h_o * std::numeric_limits<double>::epsilon();
    const int nd = tb.nd;
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < T.ne; ++r) {
        const int32_t* no = &T.enodes[3 * r];
        double* qe = &q[r * 3 * nd];
        double b[3] = {X[3 * no[0] + 2], X[3 * no[1] + 2], X[3 * no[2] + 2]};
        double ze[3], qx[3], qy[3];
        to_vertices(qe, ze);
        to_vertices(qe + nd, qx);
        to_vertices(qe + 2 * nd, qy);
        bool set_wet = true;
        for (int v = 0; v < 3; ++v)
            if (ze[v] + b[v] <= cfg.h_o + thr) {
                ze[v] = cfg.h_o - b[v];
                set_wet = false;
            }
        if (!set_wet) {
            wet[r] = 0;
            for (int v = 0; v < 3; ++v) qx[v] = qy[v] = 0.0;
            from_vertices(ze, qe, nd);
            from_vertices(qx, qe + nd, nd);
            from_vertices(qy, qe + 2 * nd, nd);
        }
    }
}

}  // namespace dgsw
