// tomato's tight-binding generator on the GPU (tomato/src/tomato_TB.F90:1-636).
//
// tomato_TB builds H (and S) of a periodic supercell from a template: the element list of
// one unit cell and its neighbours, (orbital a, orbital b, cell offset di dj dk, H_ab [, S_ab]),
// is replicated over every cell of the supercell, adding m_set_element(H, a', b', h, 1.0)
// for each (element, cell); k-point runs multiply by exp(i 2 pi k . T) with T the image's
// wrap count; a "defect" adds a scaled copy of the first atom's on-site block; and a final
// estimate of the sparsity samples num_orbs elements with the omm LCG.  The selection of the
// basis size, the supercell and the orbital cutoff from the template's info file, and the
// parsing of the files, are host work here as there.  The replication is a device kernel
// over (element, cell) pairs writing (column, row) keys and values in the reference's loop
// order; a stable device sort by key then brings each matrix element's contributions
// together in that same order, and one thread per element sums them in order, so every value
// is bit-identical to the reference's sequence of additions.  The result is a CSC matrix
// (or, for a dense label, the same matrix converted): the sorted heads come back to the host,
// where CSC handles keep their index arrays, and are compacted into column pointers there.
#include "internal.h"

#include <thrust/device_ptr.h>
#include <thrust/execution_policy.h>
#include <thrust/scan.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace ommgpu {
namespace {

struct TomatoInfo {
    int nper = 0, napc = 0, nocc = 0;
    std::vector<int> cutoffs, sizes, refs;
    std::vector<std::vector<int>> index;  // per basis size: the subset's orbital indices (1-based), or empty
};

std::vector<std::string> read_lines(const std::string& path) {
    std::ifstream f(path);
    if (!f) fail(OMM_ERR_ARG, "tomato_TB: cannot open " + path);
    std::vector<std::string> v;
    std::string ln;
    while (std::getline(f, ln)) v.push_back(ln);
    return v;
}

std::vector<long long> ints_of(const std::string& ln) {
    std::istringstream s(ln);
    std::vector<long long> v;
    long long x;
    while (s >> x) v.push_back(x);
    return v;
}

// <basedir>/<label>_template.info (tomato_TB.F90:124-180)
TomatoInfo read_info(const std::string& basedir, const std::string& label) {
    std::vector<std::string> L = read_lines(basedir + "/" + label + "_template.info");
    size_t p = 0;
    auto next = [&]() -> const std::string& {
        if (p >= L.size()) fail(OMM_ERR_ARG, "tomato_TB: template info file ends early");
        return L[p++];
    };
    auto first_int = [&](const std::string& s) {
        std::vector<long long> v = ints_of(s);
        if (v.empty()) fail(OMM_ERR_ARG, "tomato_TB: malformed template info file");
        return (int)v[0];
    };
    TomatoInfo I;
    I.nper = first_int(next());
    I.napc = first_int(next());
    I.nocc = first_int(next());
    const int ncut = first_int(next());
    for (int i = 0; i < ncut; ++i) I.cutoffs.push_back(first_int(next()));
    const int nbas = first_int(next());
    for (int i = 0; i < nbas; ++i) {
        std::vector<long long> v = ints_of(next());
        if (v.empty()) fail(OMM_ERR_ARG, "tomato_TB: malformed basis size line");
        const int sz = (int)v[0];
        I.sizes.push_back(sz);
        if (v.size() >= 2) {  // "size ref idx(1:size)": a subset of the ref-size basis (:166-174)
            const int ref = (int)v[1];
            if ((int)v.size() < 2 + sz) fail(OMM_ERR_ARG, "tomato_TB: subset index list too short");
            std::vector<int> idx(v.begin() + 2, v.begin() + 2 + sz);
            std::vector<int> full(idx);
            for (int k = 2; k <= I.napc; ++k)
                for (int l = 0; l < sz; ++l) full.push_back((k - 1) * ref + idx[l]);
            I.refs.push_back(ref);
            I.index.push_back(full);
        } else {
            I.refs.push_back(sz);
            I.index.push_back({});
        }
    }
    return I;
}

std::string element_path(const std::string& basedir, const std::string& label, int cut, int ref) {
    return basedir + "/" + label + "_" + std::to_string(cut) + "_" + std::to_string(ref) + ".template";
}

// the first record of an element file: '(2x,i10)' num_template
int read_num_template(const std::string& path) {
    std::ifstream f(path);
    if (!f) fail(OMM_ERR_ARG, "tomato_TB: cannot open " + path);
    std::string ln;
    std::getline(f, ln);
    if (ln.size() < 3) fail(OMM_ERR_ARG, "tomato_TB: malformed element file " + path);
    return std::atoi(ln.substr(2, 10).c_str());
}

// Fortran nint: nearest integer, halves away from zero
int nint_f(double x) { return x >= 0 ? (int)std::floor(x + 0.5) : -(int)std::floor(-x + 0.5); }

struct Entry {
    int o1, o2, di, dj, dk;
};

// one (element, cell) pair per thread: key = column * num_orbs + row, value (H, S), in the order
// of the reference's loops (element outermost, then cells i, j, k with k fastest)
template <bool CPLX>
__global__ void tomato_scatter_kernel(int nkept, int ncells, int n1, int n2, int n3, int nopc, int num_orbs,
                                      const int* __restrict__ el, const double* __restrict__ hv,
                                      const double* __restrict__ sv, double kx, double ky, double kz,
                                      long long* __restrict__ keys, double* __restrict__ vh,
                                      double* __restrict__ vs) {
    const long long tot = (long long)nkept * ncells;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        const int l = (int)(e / ncells), cell = (int)(e % ncells);
        const int i = cell / (n2 * n3), j = (cell / n3) % n2, k = cell % n3;
        const int o1 = el[5 * l], o2 = el[5 * l + 1], di = el[5 * l + 2], dj = el[5 * l + 3], dk = el[5 * l + 4];
        const int i2 = ((i + di) % n1 + n1) % n1, j2 = ((j + dj) % n2 + n2) % n2, k2 = ((k + dk) % n3 + n3) % n3;
        const long long a = (long long)cell * nopc + o1 - 1;
        const long long b = ((long long)(i2 * n2 + j2) * n3 + k2) * nopc + o2 - 1;
        keys[e] = b * num_orbs + a;
        if (!CPLX) {
            vh[e] = hv[l];
            if (vs) vs[e] = sv[l];
        } else {
            // wrap counts of the image, with the truncating integer division of the reference
            const int i3 = (i + di - i2) / n1, j3 = (j + dj - j2) / n2, k3 = (k + dk - k2) / n3;
            const double kt = 6.283185307179586476925286766559 * (kx * i3 + ky * j3 + kz * k3);
            double sn, cs;
            sincos(kt, &sn, &cs);
            vh[2 * e] = hv[l] * cs;
            vh[2 * e + 1] = hv[l] * sn;
            if (vs) {
                vs[2 * e] = sv[l] * cs;
                vs[2 * e + 1] = sv[l] * sn;
            }
        }
    }
}

// after the stable sort: a run of equal keys is one matrix element; its first thread sums the
// run in order and marks it (head[p] = 1)
template <int W>
__global__ void tomato_reduce_kernel(long long tot, const long long* __restrict__ keys, const long long* __restrict__ perm,
                                     const double* __restrict__ vin, double* __restrict__ vout, int* __restrict__ head) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < tot;
         p += (long long)gridDim.x * blockDim.x) {
        const bool h = p == 0 || keys[p] != keys[p - 1];
        head[p] = h ? 1 : 0;
        if (!h) continue;
        double acc[W];
#pragma unroll
        for (int q = 0; q < W; ++q) acc[q] = 0.0;
        for (long long r = p; r < tot && keys[r] == keys[p]; ++r)
#pragma unroll
            for (int q = 0; q < W; ++q) acc[q] = vin[(size_t)perm[r] * W + q] + acc[q];
#pragma unroll
        for (int q = 0; q < W; ++q) vout[(size_t)p * W + q] = acc[q];
    }
}

}  // namespace
}  // namespace ommgpu

using namespace ommgpu;

extern "C" int tomato_gpu_TB(const char* template_basedir, const char* system_label, bool switch1, double* frac_occ,
                             int* num_orbs_per_atom, bool switch2, int* num_orbs, int num_cells_dir[3], bool switch3,
                             double* sparsity, double* orb_r_cut, int* num_occ_states, bool gamma_point,
                             double k_point[3], bool defect, double defect_perturbation, msw_matrix** H,
                             msw_matrix** S, const char m_storage[5], bool build_matrix) {
    try {
        if (!template_basedir || !system_label || !frac_occ || !num_orbs_per_atom || !num_orbs || !num_cells_dir ||
            !sparsity || !orb_r_cut || !num_occ_states || !k_point)
            fail(OMM_ERR_ARG, "tomato_TB: null argument");
        const std::string base(template_basedir), label(system_label);
        const TomatoInfo I = read_info(base, label);
        if (I.sizes.empty() || I.cutoffs.empty()) fail(OMM_ERR_ARG, "tomato_TB: no basis sizes or cutoffs");
        // basis size (:184-208): the first closest frac_occ, or num_orbs_per_atom
        int ti = 0;
        if (switch1) {
            double dmin = 999999.9;
            for (size_t i = 0; i < I.sizes.size(); ++i) {
                const double d = std::fabs(*frac_occ - (double)I.nocc / (double)I.sizes[i]);
                if (d < dmin) {
                    dmin = d;
                    *num_orbs_per_atom = I.sizes[i];
                    ti = (int)i;
                }
            }
        } else {
            int j = 999999;
            const int l = *num_orbs_per_atom;
            for (size_t i = 0; i < I.sizes.size(); ++i) {
                const int k = std::abs(l - I.sizes[i]);
                if (k < j) {
                    j = k;
                    *num_orbs_per_atom = I.sizes[i];
                    ti = (int)i;
                }
            }
        }
        const int nopa = *num_orbs_per_atom, nopc = nopa * I.napc;
        *frac_occ = (double)I.nocc / (double)nopa;
        const bool is_subset = I.sizes[ti] != I.refs[ti];
        const int ref = I.refs[ti];
        // supercell (:212-245)
        int* ncd = num_cells_dir;
        if (switch2) {
            const double q = (double)*num_orbs / (double)nopc;
            ncd[0] = I.nper < 3 ? 1 : std::max(nint_f(std::pow(q, 1.0 / 3.0)), 1);
            ncd[1] = I.nper < 2 ? 1 : std::max(nint_f(std::sqrt(q / ncd[0])), 1);
            ncd[2] = I.nper < 1 ? 1 : std::max(nint_f(q / (ncd[0] * ncd[1])), 1);
        } else {
            for (int i = 0; i < 3; ++i) ncd[i] = I.nper < 3 - i ? 1 : std::max(ncd[i], 1);
        }
        const int ncells = ncd[0] * ncd[1] * ncd[2];
        if ((long long)nopc * ncells > (1LL << 30)) fail(OMM_ERR_ARG, "tomato_TB: supercell too large");
        *num_orbs = nopc * ncells;
        *num_occ_states = I.nocc * I.napc * ncells;
        const int no = *num_orbs;
        auto num_template_of = [&](int cut) {
            long long nt = read_num_template(element_path(base, label, cut, ref));
            if (is_subset) nt = nt * nopa * nopa / ((long long)ref * ref);
            return nt;
        };
        // orbital cutoff (:249-282)
        int cut_i = I.cutoffs[0];
        if (switch3) {
            double dmin = 999999.9;
            for (int c : I.cutoffs) {
                const double d2 = std::max(1.0 - (double)num_template_of(c) * ncells / ((double)no * no), 0.0);
                const double d = std::fabs(*sparsity - d2);
                if (d < dmin) {
                    dmin = d;
                    cut_i = c;
                }
            }
        } else {
            int j = 999999;
            const int l = nint_f(*orb_r_cut * 100.0);
            for (int c : I.cutoffs) {
                const int k = std::abs(l - c);
                if (k < j) {
                    j = k;
                    cut_i = c;
                }
            }
        }
        *orb_r_cut = cut_i * 0.01;
        for (int d = 0; d < 3; ++d)  // no k points in non-periodic directions (:305-307)
            if (I.nper < 3 - d) k_point[d] = 0.0;
        if (!build_matrix) {
            *sparsity = std::max(1.0 - (double)num_template_of(cut_i) * ncells / ((double)no * no), 0.0);
            if (H) *H = nullptr;
            if (S) *S = nullptr;
            set_last_error("");
            return OMM_OK;
        }
        if (!H || !S || !m_storage) fail(OMM_ERR_ARG, "tomato_TB: null matrix handle or label");
        const Label lab = parse_storage(m_storage);
        if (lab.real != gamma_point) fail(OMM_ERR_ARG, "tomato_TB: a Gamma-point run needs a real label, k points complex");
        // the element file (:339-378)
        const std::string path = element_path(base, label, cut_i, ref);
        std::vector<std::string> L = read_lines(path);
        if (L.empty()) fail(OMM_ERR_ARG, "tomato_TB: empty element file " + path);
        const int num = std::atoi(L[0].size() > 2 ? L[0].substr(2, 10).c_str() : "0");
        if (num < 0 || (int)L.size() < 1 + num) fail(OMM_ERR_ARG, "tomato_TB: element file shorter than its count");
        std::vector<Entry> ti_(num);
        std::vector<double> hv(num), sv(num);
        bool overlap = false;
        for (int l = 0; l < num; ++l) {
            std::string s = L[1 + l];
            for (char& ch : s)
                if (ch == 'D' || ch == 'd') ch = 'E';
            std::istringstream in(s);
            Entry e{};
            double h = 0.0, sval = 0.0;
            if (!(in >> e.o1 >> e.o2 >> e.di >> e.dj >> e.dk >> h)) fail(OMM_ERR_ARG, "tomato_TB: malformed element line");
            const bool has_s = (bool)(in >> sval);
            if (l == 0) overlap = has_s;
            ti_[l] = e;
            hv[l] = h;
            sv[l] = has_s ? sval : 0.0;
        }
        // the elements kept (a subset basis keeps those of its orbitals, renumbered, :400-408)
        std::vector<int> conv;
        if (is_subset) {
            conv.assign((size_t)I.napc * ref + 1, 0);
            for (int i = 0; i < nopc; ++i) conv[I.index[ti][i]] = i + 1;
        }
        auto mapped = [&](const Entry& e, int& a, int& b) {
            a = e.o1;
            b = e.o2;
            if (!is_subset) return a >= 1 && a <= nopc && b >= 1 && b <= nopc;
            if (a < 1 || b < 1 || a >= (int)conv.size() || b >= (int)conv.size() || !conv[a] || !conv[b]) return false;
            a = conv[a];
            b = conv[b];
            return true;
        };
        std::vector<int> el;
        std::vector<double> kh, ks;
        for (int l = 0; l < num; ++l) {
            int a, b;
            if (!mapped(ti_[l], a, b)) continue;
            el.insert(el.end(), {a, b, ti_[l].di, ti_[l].dj, ti_[l].dk});
            kh.push_back(hv[l]);
            ks.push_back(sv[l]);
        }
        // the defect: the first atom's cell-0 elements, scaled, added after the supercell (:425-436)
        std::vector<long long> dkey;
        std::vector<double> dval;
        if (defect)
            for (int l = 0; l < num; ++l) {
                int a, b;
                const Entry& e = ti_[l];
                if (!mapped(e, a, b)) continue;
                if (a <= nopa && b <= nopa && e.di == 0 && e.dj == 0 && e.dk == 0) {
                    dkey.push_back((long long)(b - 1) * no + (a - 1));
                    dval.push_back(defect_perturbation * hv[l]);
                }
            }
        const int nkept = (int)kh.size();
        const int W = gamma_point ? 1 : 2;
        const long long nmain = (long long)nkept * ncells, tot = nmain + (long long)dkey.size();
        cudaStream_t st = rt().stream;
        DevBuf d_el, d_hv, d_sv, d_keys, d_perm, d_vh, d_vs, d_oh, d_os, d_head;
        d_el.alloc(std::max<size_t>(el.size(), 1) * sizeof(int));
        d_hv.alloc(std::max<size_t>(kh.size(), 1) * sizeof(double));
        d_sv.alloc(std::max<size_t>(ks.size(), 1) * sizeof(double));
        d_keys.alloc(std::max<long long>(tot, 1) * sizeof(long long));
        d_perm.alloc(std::max<long long>(tot, 1) * sizeof(long long));
        d_vh.alloc(std::max<long long>(tot, 1) * W * sizeof(double));
        if (overlap) d_vs.alloc(std::max<long long>(tot, 1) * W * sizeof(double));
        if (!el.empty()) {
            OMM_CK(cudaMemcpyAsync(d_el.p, el.data(), el.size() * sizeof(int), cudaMemcpyHostToDevice, st));
            OMM_CK(cudaMemcpyAsync(d_hv.p, kh.data(), kh.size() * sizeof(double), cudaMemcpyHostToDevice, st));
            OMM_CK(cudaMemcpyAsync(d_sv.p, ks.data(), ks.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        if (nmain > 0) {
            const int grid = (int)std::min<long long>((nmain + 255) / 256, 148LL * 32);
            if (gamma_point)
                tomato_scatter_kernel<false><<<grid, 256, 0, st>>>(
                    nkept, ncells, ncd[0], ncd[1], ncd[2], nopc, no, d_el.as<int>(), d_hv.as<double>(),
                    d_sv.as<double>(), 0.0, 0.0, 0.0, d_keys.as<long long>(), d_vh.as<double>(),
                    overlap ? d_vs.as<double>() : nullptr);
            else
                tomato_scatter_kernel<true><<<grid, 256, 0, st>>>(
                    nkept, ncells, ncd[0], ncd[1], ncd[2], nopc, no, d_el.as<int>(), d_hv.as<double>(),
                    d_sv.as<double>(), k_point[0], k_point[1], k_point[2], d_keys.as<long long>(), d_vh.as<double>(),
                    overlap ? d_vs.as<double>() : nullptr);
            OMM_KCHECK();
        }
        if (!dkey.empty()) {  // defect entries after the supercell's, H only (real part for k points)
            std::vector<double> dv((size_t)dkey.size() * W, 0.0), zs((size_t)dkey.size() * W, 0.0);
            for (size_t q = 0; q < dkey.size(); ++q) dv[q * W] = dval[q];
            OMM_CK(cudaMemcpyAsync(d_keys.as<long long>() + nmain, dkey.data(), dkey.size() * sizeof(long long),
                                   cudaMemcpyHostToDevice, st));
            OMM_CK(cudaMemcpyAsync(d_vh.as<double>() + nmain * W, dv.data(), dv.size() * sizeof(double),
                                   cudaMemcpyHostToDevice, st));
            if (overlap)
                OMM_CK(cudaMemcpyAsync(d_vs.as<double>() + nmain * W, zs.data(), zs.size() * sizeof(double),
                                       cudaMemcpyHostToDevice, st));
            OMM_CK(cudaStreamSynchronize(st));  // the host vectors go out of scope
        }
        // stable sort of the keys: each element's contributions together, in the reference's order
        thrust::device_ptr<long long> kp(d_keys.as<long long>()), pp(d_perm.as<long long>());
        thrust::sequence(thrust::cuda::par.on(st), pp, pp + tot);
        thrust::stable_sort_by_key(thrust::cuda::par.on(st), kp, kp + tot, pp);
        d_head.alloc(std::max<long long>(tot, 1) * sizeof(int));
        d_oh.alloc(std::max<long long>(tot, 1) * W * sizeof(double));
        if (overlap) d_os.alloc(std::max<long long>(tot, 1) * W * sizeof(double));
        const int rgrid = (int)std::min<long long>((tot + 255) / 256, 148LL * 32);
        if (tot > 0) {
            if (W == 1) {
                tomato_reduce_kernel<1><<<rgrid, 256, 0, st>>>(tot, d_keys.as<long long>(), d_perm.as<long long>(),
                                                               d_vh.as<double>(), d_oh.as<double>(), d_head.as<int>());
                OMM_KCHECK();
                if (overlap) {
                    tomato_reduce_kernel<1><<<rgrid, 256, 0, st>>>(tot, d_keys.as<long long>(), d_perm.as<long long>(),
                                                                   d_vs.as<double>(), d_os.as<double>(), d_head.as<int>());
                    OMM_KCHECK();
                }
            } else {
                tomato_reduce_kernel<2><<<rgrid, 256, 0, st>>>(tot, d_keys.as<long long>(), d_perm.as<long long>(),
                                                               d_vh.as<double>(), d_oh.as<double>(), d_head.as<int>());
                OMM_KCHECK();
                if (overlap) {
                    tomato_reduce_kernel<2><<<rgrid, 256, 0, st>>>(tot, d_keys.as<long long>(), d_perm.as<long long>(),
                                                                   d_vs.as<double>(), d_os.as<double>(), d_head.as<int>());
                    OMM_KCHECK();
                }
            }
        }
        // the heads (one per matrix element) to the host: CSC arrays of both matrices (same pattern)
        std::vector<long long> keys(tot);
        std::vector<int> heads(tot);
        std::vector<double> oh((size_t)tot * W), os(overlap ? (size_t)tot * W : 0);
        if (tot > 0) {
            OMM_CK(cudaMemcpyAsync(keys.data(), d_keys.p, tot * sizeof(long long), cudaMemcpyDeviceToHost, st));
            OMM_CK(cudaMemcpyAsync(heads.data(), d_head.p, tot * sizeof(int), cudaMemcpyDeviceToHost, st));
            OMM_CK(cudaMemcpyAsync(oh.data(), d_oh.p, oh.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
            if (overlap)
                OMM_CK(cudaMemcpyAsync(os.data(), d_os.p, os.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
        OMM_CK(cudaStreamSynchronize(st));
        std::vector<int> colptr(no + 1, 0), rowind;
        std::vector<double> vh, vs;
        for (long long p = 0; p < tot; ++p) {
            if (!heads[p]) continue;
            const int c = (int)(keys[p] / no), r = (int)(keys[p] % no);
            colptr[c + 1]++;
            rowind.push_back(r);
            for (int q = 0; q < W; ++q) vh.push_back(oh[(size_t)p * W + q]);
            if (overlap)
                for (int q = 0; q < W; ++q) vs.push_back(os[(size_t)p * W + q]);
        }
        for (int j = 0; j < no; ++j) colptr[j + 1] += colptr[j];
        const int nnz = (int)rowind.size();
        // the sparsity estimate (:560-580): num_orbs LCG-sampled elements of H, the fraction that
        // are zero (the NORAND seed 123456 of omm_rand_seed)
        auto get = [&](int a, int b) {  // 1-based element of H
            if (a < 1 || b < 1 || a > no || b > no) return true;
            const int* lo = rowind.data() + colptr[b - 1];
            const int* hi = rowind.data() + colptr[b];
            const int* it = std::lower_bound(lo, hi, a - 1);
            if (it == hi || *it != a - 1) return true;
            const size_t k = (size_t)(it - rowind.data());
            return W == 1 ? vh[k] == 0.0 : (vh[2 * k] == 0.0 && vh[2 * k + 1] == 0.0);
        };
        long long seed = 123456, nz = 0;
        const long long m31 = 1LL << 31;
        for (int i = 0; i < no; ++i) {
            seed = (1103515245LL * seed + 12345) % m31;
            const int a = (int)std::ceil(no * ((double)seed / (double)m31));
            seed = (1103515245LL * seed + 12345) % m31;
            const int b = (int)std::ceil(no * ((double)seed / (double)m31));
            if (get(a, b)) ++nz;
        }
        *sparsity = (double)nz / (double)no;
        // the matrices in the requested storage: CSC, or converted to the dense label
        char csc_label[6];
        std::snprintf(csc_label, sizeof csc_label, "%c%c%s", m_storage[0] == 's' ? 's' : (m_storage[0] == 'p' ? 'p' : 'g'),
                      m_storage[1], "csc");
        auto make = [&](const std::vector<double>& v, msw_matrix** out) {
            msw_matrix* M = nullptr;
            int rc = msw_register_csc(&M, csc_label, no, no, nnz, colptr.data(), rowind.data(), v.data(), 0);
            if (rc < 0) throw Error{rc, omm_gpu_last_error()};
            if (lab.fmt == Fmt::CSC) {
                *out = M;
                return;
            }
            msw_matrix* Dn = nullptr;
            rc = msw_copy(&Dn, M, m_storage);
            msw_deallocate(&M);
            if (rc < 0) throw Error{rc, omm_gpu_last_error()};
            *out = Dn;
        };
        make(vh, H);
        if (overlap) make(vs, S);
        else *S = nullptr;  // no overlap in the template: S is not allocated (:380)
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    }
    set_last_error("");
    return OMM_OK;
}
