// Host-side Hamiltonian builder: neighbour shells, DMI vectors, coupling blocks.
//
// The steps follow Matjes' set-up path so that the couplings are the ones the
// reference would hand to its sparse backend (paths relative to src/):
//   shells by sorted distance, 0-distance counted for equal types, eps =
//   1e-7 * min|a_i| .............................. setup/neighbor_type.f90:182-330
//   pairs unfolded with the open-boundary cut ...... setup/neighbor_type.f90:135-180
//   J block  c_H_J * J * I ....................... Energy/exchange_Heisenberg_J.f90:78-124
//   DMI block c_H_D * D * [d]x, d from the mediator
//   atoms nearest the bond centre ................ Energy/exchange_Heisenberg_D.f90:79-132, 253-330
//   anisotropy c_H_ani * K e e^T .................. Energy/anisotropy_heisenberg.f90:243-292
//   every local block thinned by |h| > 1e-10 max|h| Energy/setH_util.f90:10-36
//   dipolar K(r) on the N_rep grid with images .... Energy/dipolar_magnetic.f90:58-177, 275-308
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <numeric>

#include "mj_internal.hpp"

namespace mj {
namespace {

inline double norm3(const double* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
inline void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

double shell_eps(const Geometry& g) {
    double e = 1e300;
    for (int j = 0; j < 3; ++j) e = std::min(e, norm3(g.d.areal[j]));
    return e * 1.0e-7;
}

void lattice_shift(const Geometry& g, int i1, int i2, int i3, double out[3]) {
    for (int k = 0; k < 3; ++k) out[k] = i1 * g.d.areal[0][k] + i2 * g.d.areal[1][k] + i3 * g.d.areal[2][k];
}

struct Candidate {
    double dist;
    int a1, a2;
    int o[3];
};

// The (atom, atom, cell offset) connections forming shell `rank` (1 = nearest).
bool shell_connections(const Geometry& g, int t1, int t2, int rank, std::vector<Candidate>& out, std::string& err) {
    std::vector<int> id1, id2;
    for (int a = 0; a < g.d.natom; ++a) {
        if (g.d.attype[a] == t1) id1.push_back(a);
        if (g.d.attype[a] == t2) id2.push_back(a);
    }
    if (id1.empty() || id2.empty()) {
        err = "no atom of type " + std::to_string(id1.empty() ? t1 : t2) + " in the cell";
        return false;
    }
    const int want = rank + (t1 == t2 ? 1 : 0);
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        const bool active = g.d.L[d] > 1 || g.d.periodic[d];
        lo[d] = active ? -want : 0;
        hi[d] = active ? want : 0;
    }
    std::vector<Candidate> all;
    for (int i3 = lo[2]; i3 <= hi[2]; ++i3)
        for (int i2 = lo[1]; i2 <= hi[1]; ++i2)
            for (int i1 = lo[0]; i1 <= hi[0]; ++i1) {
                double sh[3];
                lattice_shift(g, i1, i2, i3, sh);
                for (int b : id2)
                    for (int a : id1) {
                        double v[3];
                        for (int k = 0; k < 3; ++k) v[k] = g.pos[b][k] - g.pos[a][k] + sh[k];
                        all.push_back({norm3(v), a, b, {i1, i2, i3}});
                    }
            }
    std::stable_sort(all.begin(), all.end(), [](const Candidate& x, const Candidate& y) { return x.dist < y.dist; });
    const double eps = shell_eps(g);
    // walk the distance groups; a group opens when d exceeds its first member + eps
    size_t begin = all.size(), end = all.size();
    int group = 0;
    double first = -10.0 * eps;
    for (size_t i = 0; i < all.size(); ++i) {
        if (all[i].dist > first + eps) {
            ++group;
            first = all[i].dist;
            if (group == want) begin = i;
            if (group == want + 1) {
                end = i;
                break;
            }
        }
    }
    if (begin == all.size()) {
        err = "shell " + std::to_string(rank) + " not found for types " + std::to_string(t1) + "," + std::to_string(t2);
        return false;
    }
    out.assign(all.begin() + begin, all.begin() + end);
    return true;
}

// DMI vector of one connection: normalised sum over the mediator atoms closest to
// the bond centre of normalise((r_a - r_n) x (r_b - r_n)).
bool dmi_vector(const Geometry& g, const Candidate& c, int tmed, double dmi[3], std::string& err) {
    double ra[3], rb[3], cen[3], sh[3];
    lattice_shift(g, c.o[0], c.o[1], c.o[2], sh);
    for (int k = 0; k < 3; ++k) {
        ra[k] = g.pos[c.a1][k];
        rb[k] = g.pos[c.a2][k] + sh[k];
        cen[k] = (ra[k] + rb[k]) * 0.5;
    }
    // centre folded into the first cell through fractional coordinates
    const double* a1 = g.d.areal[0];
    const double* a2 = g.d.areal[1];
    const double* a3 = g.d.areal[2];
    double b1[3], b2[3], b3[3];
    cross3(a2, a3, b1);
    cross3(a3, a1, b2);
    cross3(a1, a2, b3);
    const double vol = a1[0] * b1[0] + a1[1] * b1[1] + a1[2] * b1[2];
    const double f1 = std::floor((cen[0] * b1[0] + cen[1] * b1[1] + cen[2] * b1[2]) / vol);
    const double f2 = std::floor((cen[0] * b2[0] + cen[1] * b2[1] + cen[2] * b2[2]) / vol);
    const double f3 = std::floor((cen[0] * b3[0] + cen[1] * b3[1] + cen[2] * b3[2]) / vol);
    double cuc[3];
    for (int k = 0; k < 3; ++k) cuc[k] = cen[k] - f1 * a1[k] - f2 * a2[k] - f3 * a3[k];
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        const bool active = g.d.L[d] > 1 || g.d.periodic[d];
        lo[d] = active ? -1 : 0;
        hi[d] = active ? 1 : 0;
    }
    struct Med { double dist; double p[3]; };
    std::vector<Med> meds;
    for (int i3 = lo[2]; i3 <= hi[2]; ++i3)
        for (int i2 = lo[1]; i2 <= hi[1]; ++i2)
            for (int i1 = lo[0]; i1 <= hi[0]; ++i1) {
                double s2[3];
                lattice_shift(g, i1, i2, i3, s2);
                for (int a = 0; a < g.d.natom; ++a) {
                    if (g.d.attype[a] != tmed) continue;
                    Med m;
                    double v[3];
                    for (int k = 0; k < 3; ++k) {
                        v[k] = g.pos[a][k] - cuc[k] + s2[k];
                        m.p[k] = g.pos[a][k] + s2[k] - cuc[k] + cen[k];
                    }
                    m.dist = norm3(v);
                    meds.push_back(m);
                }
            }
    if (meds.empty()) {
        err = "no mediator atom of type " + std::to_string(tmed);
        return false;
    }
    double best = 1e300;
    for (const Med& m : meds) best = std::min(best, m.dist);
    const double eps = shell_eps(g);
    double sum[3] = {0.0, 0.0, 0.0};
    for (const Med& m : meds) {
        if (!(m.dist <= best + eps)) continue;
        double d1[3], d2[3], cr[3];
        for (int k = 0; k < 3; ++k) {
            d1[k] = ra[k] - m.p[k];
            d2[k] = rb[k] - m.p[k];
        }
        cross3(d1, d2, cr);
        const double n = norm3(cr);
        if (n > 1e-8)
            for (int k = 0; k < 3; ++k) sum[k] += cr[k] / n;
    }
    const double n = norm3(sum);
    if (n > 1e-8)
        for (int k = 0; k < 3; ++k) sum[k] /= n;
    std::memcpy(dmi, sum, sizeof(sum));
    return true;
}

// get_coo thinning of one local 3x3 block (the only non-zero block of the term)
void thin_block(double* T, double maxv) {
    const double thres = maxv * 1.0e-10;
    for (int k = 0; k < 9; ++k)
        if (!(std::fabs(T[k]) > thres)) T[k] = 0.0;
}

void add_block(std::vector<Block>& blocks, int a, int b, const int o[3], const double* T) {
    for (Block& x : blocks) {
        if (x.a == a && x.b == b && x.o[0] == o[0] && x.o[1] == o[1] && x.o[2] == o[2]) {
            for (int k = 0; k < 9; ++k) x.T[k] = x.T[k] + T[k];
            return;
        }
    }
    Block nb;
    nb.a = a;
    nb.b = b;
    std::memcpy(nb.o, o, sizeof(nb.o));
    std::memcpy(nb.T, T, sizeof(nb.T));
    blocks.push_back(nb);
}

}  // namespace

bool build_geometry(const mj_lattice_desc& lat, Geometry& g, std::string& err) {
    g.d = lat;
    if (lat.natom < 1 || lat.natom > MJ_MAX_ATOMS) {
        err = "natom out of range";
        return false;
    }
    for (int d = 0; d < 3; ++d)
        if (lat.L[d] < 1) {
            err = "lattice dimensions must be >= 1";
            return false;
        }
    g.nmag = 0;
    for (int a = 0; a < lat.natom; ++a) {
        for (int k = 0; k < 3; ++k)
            g.pos[a][k] = lat.frac[a][0] * lat.areal[0][k] + lat.frac[a][1] * lat.areal[1][k] + lat.frac[a][2] * lat.areal[2][k];
        if (lat.moment[a] > 0.0) {
            g.magidx[a] = g.nmag;
            g.magatom[g.nmag] = a;
            ++g.nmag;
        } else {
            g.magidx[a] = -1;
        }
    }
    if (g.nmag == 0) {
        err = "no magnetic atom in the cell";
        return false;
    }
    return true;
}

bool build_blocks(const Geometry& g, const mj_hamiltonian_desc& h, std::vector<Block>& blocks,
                  std::vector<double>& onsite, std::string& err) {
    blocks.clear();
    const int nm = g.nmag;
    onsite.assign(static_cast<size_t>(9) * nm * nm, 0.0);
    for (int t = 0; t < h.nJ; ++t) {
        std::vector<Candidate> sh;
        if (!shell_connections(g, h.J[t].t1, h.J[t].t2, h.J[t].shell, sh, err)) return false;
        for (const Candidate& c : sh) {
            const int a = g.magidx[c.a1], b = g.magidx[c.a2];
            if (a < 0 || b < 0) continue;
            double T[9] = {0};
            const double v = h.c_H_J * h.J[t].value;
            T[0] = T[4] = T[8] = v;
            thin_block(T, std::fabs(v));
            if (v != 0.0) add_block(blocks, a, b, c.o, T);
        }
    }
    for (int t = 0; t < h.nD; ++t) {
        std::vector<Candidate> sh;
        if (!shell_connections(g, h.D[t].t1, h.D[t].t2, h.D[t].shell, sh, err)) return false;
        bool any = false;
        for (const Candidate& c : sh) {
            double d[3];
            if (!dmi_vector(g, c, h.D[t].tmed, d, err)) return false;
            if (!(norm3(d) > 1e-8)) continue;
            const int a = g.magidx[c.a1], b = g.magidx[c.a2];
            if (a < 0 || b < 0) continue;
            any = true;
            const double D = h.D[t].value;
            // m_a^T T m_b = c_H_D * D * d . (m_a x m_b)
            double T[9] = {0};
            T[0 * 3 + 1] = h.c_H_D * (d[2] * D);
            T[2 * 3 + 0] = h.c_H_D * (d[1] * D);
            T[1 * 3 + 2] = h.c_H_D * (d[0] * D);
            T[1 * 3 + 0] = h.c_H_D * (-d[2] * D);
            T[0 * 3 + 2] = h.c_H_D * (-d[1] * D);
            T[2 * 3 + 1] = h.c_H_D * (-d[0] * D);
            double mx = 0.0;
            for (double x : T) mx = std::max(mx, std::fabs(x));
            thin_block(T, mx);
            add_block(blocks, a, b, c.o, T);
        }
        if (!any) {
            err = "no DMI contribution found (mediator geometry gives d = 0)";
            return false;
        }
    }
    if (h.nK > 0) {
        // all anisotropy inputs accumulate into one cell matrix before thinning
        const int dm = 3 * nm;
        std::vector<double> H(static_cast<size_t>(dm) * dm, 0.0);
        for (int t = 0; t < h.nK; ++t) {
            const double n = norm3(h.K[t].axis);
            if (!(n > 0.0)) {
                err = "anisotropy axis has zero length";
                return false;
            }
            const double e[3] = {h.K[t].axis[0] / n, h.K[t].axis[1] / n, h.K[t].axis[2] / n};
            for (int a = 0; a < g.d.natom; ++a) {
                if (g.d.attype[a] != h.K[t].type || g.magidx[a] < 0) continue;
                const int o = 3 * g.magidx[a];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j)
                        H[(o + i) * dm + o + j] = H[(o + i) * dm + o + j] + h.K[t].value * e[i] * e[j];
            }
        }
        double mx = 0.0;
        for (double& x : H) {
            x = x * h.c_H_ani;
            mx = std::max(mx, std::fabs(x));
        }
        for (double& x : H)
            if (!(std::fabs(x) > mx * 1.0e-10)) x = 0.0;
        for (int a = 0; a < nm; ++a)
            for (int b = 0; b < nm; ++b)
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j)
                        onsite[(static_cast<size_t>(a) * nm + b) * 9 + 3 * i + j] = H[(3 * a + i) * dm + 3 * b + j];
    }
    return true;
}

void build_noise_tables(double* tab) {
    // evaluated in extended precision, then rounded once to double
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int i = 0; i < 1024; ++i) {
        const long double a = two_pi * (static_cast<long double>(i) + 0.5L) / 1024.0L;
        tab[2 * i] = static_cast<double>(sinl(a));
        tab[2 * i + 1] = static_cast<double>(cosl(a));
    }
    for (int j = 0; j < 1024; ++j) {
        const long double F = 1.0L + (static_cast<long double>(j) + 0.5L) / 1024.0L;
        tab[2048 + 2 * j] = static_cast<double>(1.0L / F);
        tab[2048 + 2 * j + 1] = static_cast<double>(logl(F));
    }
}

bool build_dipolar_kernel(const Geometry& g, const mj_hamiltonian_desc& h, int nrep[3], std::vector<double>& K,
                          std::string& err) {
    if (g.nmag != 1) {
        err = "the FFT dipolar kernel supports one magnetic atom per cell";
        return false;
    }
    // grid rule: dip_on 1 is the reference's (Hamiltonian_type/fft_ham_base.f90:204-214,
    // open axes doubled, periodic axes kept with their images folded in circularly);
    // dip_on 2 zero-pads every axis longer than one cell to 2 L, so that the
    // convolution is linear and each pair's image sum runs over the symmetric
    // window -cut..cut (the explicit route of Energy/dipolar_magnetic.f90:181-273)
    const bool full = h.dip_on == 2;
    int kb0[3], kb1[3];
    for (int d = 0; d < 3; ++d) {
        const bool keep = g.d.L[d] == 1 || (g.d.periodic[d] && !full);
        nrep[d] = keep ? g.d.L[d] : 2 * g.d.L[d];
        kb0[d] = keep ? 0 : -g.d.L[d] + 1;
        kb1[d] = g.d.L[d] - 1;
    }
    const int64_t nk = static_cast<int64_t>(nrep[0]) * nrep[1] * nrep[2];
    K.assign(static_cast<size_t>(nk) * 9, 0.0);
    // periodic images of the super-cell, only along truly periodic axes
    std::vector<std::array<double, 3>> images;
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = g.d.periodic[d] ? -h.dip_period_cut[d] : 0;
        hi[d] = g.d.periodic[d] ? h.dip_period_cut[d] : 0;
    }
    for (int i3 = lo[2]; i3 <= hi[2]; ++i3)
        for (int i2 = lo[1]; i2 <= hi[1]; ++i2)
            for (int i1 = lo[0]; i1 <= hi[0]; ++i1) {
                std::array<double, 3> v;
                for (int k = 0; k < 3; ++k)
                    v[k] = g.d.areal[0][k] * g.d.L[0] * static_cast<double>(i1) +
                           g.d.areal[1][k] * g.d.L[1] * static_cast<double>(i2) +
                           g.d.areal[2][k] * g.d.L[2] * static_cast<double>(i3);
                images.push_back(v);
            }
    const double mu = g.d.moment[g.magatom[0]];
    for (int i3 = kb0[2]; i3 <= kb1[2]; ++i3) {
        const int m3 = ((i3 % nrep[2]) + nrep[2]) % nrep[2];
        for (int i2 = kb0[1]; i2 <= kb1[1]; ++i2) {
            const int m2 = ((i2 % nrep[1]) + nrep[1]) % nrep[1];
            for (int i1 = kb0[0]; i1 <= kb1[0]; ++i1) {
                const int m1 = ((i1 % nrep[0]) + nrep[0]) % nrep[0];
                const int64_t ik = m1 + static_cast<int64_t>(nrep[0]) * (m2 + static_cast<int64_t>(nrep[1]) * m3);
                double base[3];
                lattice_shift(g, i1, i2, i3, base);
                double acc[9] = {0};
                for (const auto& im : images) {
                    const double df[3] = {base[0] + im[0], base[1] + im[1], base[2] + im[2]};
                    const double r = norm3(df);
                    if (r == 0.0) continue;  // self term vanishes
                    const double u[3] = {df[0] / r, df[1] / r, df[2] / r};
                    const double r3 = r * r * r;
                    for (int a = 0; a < 3; ++a)
                        for (int b = 0; b < 3; ++b) acc[3 * a + b] += (3.0 * u[a] * u[b] - (a == b ? 1.0 : 0.0)) / r3;
                }
                for (int q = 0; q < 9; ++q) {
                    const double v = acc[q] * (mu * mu);
                    K[static_cast<size_t>(ik) * 9 + q] = -v * kDipPref * 0.5 * 0.25 / kPi;
                }
            }
        }
    }
    return true;
}

}  // namespace mj
