// Handle construction: k-distribution, cloud LUTs and band discretisation.
//
// Host-side restatement of the table preparation in the reference constructors
// (src/Gas_optics_rrtmgp.cpp:53-363 helpers, :391-742 ctors and init_abs_coeffs;
// src/Cloud_optics.cpp:29-69), producing g-point-fastest device tables in FP32 and FP64.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "common.cuh"

namespace rrtmgp_b200 {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int status, const std::string& msg)
{
    g_last_error = msg;
    return status;
}

int cuda_status(cudaError_t err, const char* where)
{
    g_last_error = std::string(where) + ": " + cudaGetErrorString(err);
    return RRTMGP_B200_ERR_CUDA;
}

namespace {

std::string trim(const char* c)
{
    if (!c) return "";
    std::string s(c);
    const size_t a = s.find_first_not_of(" \t\n\r");
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(" \t\n\r");
    return s.substr(a, b - a + 1);
}

// 1-based position of s in v, -1 if absent (find_index, Gas_optics_rrtmgp.cpp:43-51).
int find1(const std::vector<std::string>& v, const std::string& s)
{
    for (size_t i = 0; i < v.size(); ++i)
        if (v[i] == s) return int(i) + 1;
    return -1;
}

// Packs host arrays into one device allocation (256-byte aligned sub-buffers).
struct Arena {
    std::vector<char> host;
    std::vector<std::pair<size_t, void**>> fixups;

    template <typename U>
    void add(const std::vector<U>& v, const U** dst)
    {
        size_t off = (host.size() + 255) & ~size_t(255);
        host.resize(off + std::max<size_t>(v.size(), 1) * sizeof(U), 0);
        if (!v.empty()) std::memcpy(host.data() + off, v.data(), v.size() * sizeof(U));
        fixups.push_back({off, reinterpret_cast<void**>(const_cast<U**>(dst))});
    }

    int upload(std::vector<void*>& allocs)
    {
        void* d = nullptr;
        if (cudaMalloc(&d, std::max<size_t>(host.size(), 256)) != cudaSuccess)
            return fail(RRTMGP_B200_ERR_ALLOC, "cudaMalloc of k-distribution tables failed");
        RB_CUDA(cudaMemcpy(d, host.data(), host.size(), cudaMemcpyHostToDevice), "table upload");
        allocs.push_back(d);
        for (auto& f : fixups) *f.second = static_cast<char*>(d) + f.first;
        return RRTMGP_B200_OK;
    }
};

template <typename T>
std::vector<T> conv(const double* p, size_t n)
{
    std::vector<T> out(n);
    for (size_t i = 0; i < n; ++i) out[i] = T(p[i]);
    return out;
}

struct MinorHost {
    std::vector<int> gstart, gend, kstart, flav, gas, sgas, flags;
    std::vector<double> kminor;  // [ntemp][neta][ncontrib_red]
    int ncontrib = 0;
    std::vector<int> band_begin, band_list;
};

int bands_init(rrtmgp_b200_bands_t& b, int nband, const int* lims)
{
    RB_CHECK_ARG(nband > 0 && lims, "bands: nband must be > 0");
    b.nband = nband;
    b.band_lims_host.assign(lims, lims + 2 * nband);
    int ngpt = 0;
    for (int i = 0; i < nband; ++i) {
        RB_CHECK_ARG(lims[2 * i] >= 1 && lims[2 * i + 1] >= lims[2 * i], "bands: bad g-point limits");
        ngpt = std::max(ngpt, lims[2 * i + 1]);
    }
    b.ngpt = ngpt;
    std::vector<int> bl(2 * nband), g2b(ngpt, 0);
    for (int i = 0; i < nband; ++i) {
        bl[2 * i] = lims[2 * i] - 1;
        bl[2 * i + 1] = lims[2 * i + 1];
        for (int g = lims[2 * i] - 1; g < lims[2 * i + 1]; ++g) g2b[g] = i;
    }
    if (cudaMalloc(&b.d_band_lims, bl.size() * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b.d_gpt2band, g2b.size() * sizeof(int)) != cudaSuccess)
        return fail(RRTMGP_B200_ERR_ALLOC, "cudaMalloc of band tables failed");
    RB_CUDA(cudaMemcpy(b.d_band_lims, bl.data(), bl.size() * sizeof(int), cudaMemcpyHostToDevice), "bands upload");
    RB_CUDA(cudaMemcpy(b.d_gpt2band, g2b.data(), g2b.size() * sizeof(int), cudaMemcpyHostToDevice), "bands upload");
    return RRTMGP_B200_OK;
}

void bands_free(rrtmgp_b200_bands_t& b)
{
    if (b.d_band_lims) cudaFree(b.d_band_lims);
    if (b.d_gpt2band) cudaFree(b.d_gpt2band);
    b.d_band_lims = b.d_gpt2band = nullptr;
}

template <typename T>
int fill_view(rrtmgp_b200_kdist_t* k, KdistView<T>& v, const rrtmgp_b200_kdist_tables* t,
              const std::vector<double>& vmr_red, const std::vector<int>& flavor,
              const std::vector<int>& band_flav, const MinorHost* mh)
{
    const size_t nk = size_t(t->ntemp) * (t->npres + 1) * t->neta * t->ngpt;
    const auto& info = k->info;
    v.ngas = info.ngas; v.nband = t->nband; v.ngpt = t->ngpt; v.ntemp = t->ntemp;
    v.npres = t->npres; v.neta = t->neta; v.nflav = info.nflav; v.nplanck = t->nplanck_temp;
    v.idx_h2o = find1(k->gas_names, "h2o");
    v.has_rayleigh = info.has_rayleigh;
    v.is_lw = info.is_longwave;
    const double pmin = t->press_ref[t->npres - 1], pmax = t->press_ref[0];
    v.press_ref_log0 = T(std::log(t->press_ref[0]));
    v.press_ref_log_delta = T((std::log(pmin) - std::log(pmax)) / (t->npres - 1));
    v.press_ref_trop_log = T(std::log(t->press_ref_trop));
    v.temp_ref_min = T(t->temp_ref[0]);
    v.temp_ref_delta = T((t->temp_ref[t->ntemp - 1] - t->temp_ref[0]) / (t->ntemp - 1));
    v.totplnk_delta = t->nplanck_temp > 1
        ? T((t->temp_ref[t->ntemp - 1] - t->temp_ref[0]) / (t->nplanck_temp - 1)) : T(0);

    Arena a;
    std::vector<T> temp_ref = conv<T>(t->temp_ref, t->ntemp);
    std::vector<T> vmr = conv<T>(vmr_red.data(), vmr_red.size());
    a.add(temp_ref, &v.temp_ref);
    a.add(vmr, &v.vmr_ref);
    a.add(flavor, &v.flavor);
    a.add(band_flav, &v.band_flav);
    std::vector<int> bl(2 * t->nband), g2b(t->ngpt);
    for (int b = 0; b < t->nband; ++b) {
        bl[2 * b] = t->band_lims_gpt[2 * b] - 1;
        bl[2 * b + 1] = t->band_lims_gpt[2 * b + 1];
        for (int g = bl[2 * b]; g < bl[2 * b + 1]; ++g) g2b[g] = b;
    }
    a.add(bl, &v.band_lims);
    a.add(g2b, &v.gpt2band);
    std::vector<T> kmaj = conv<T>(t->kmajor, nk);
    a.add(kmaj, &v.kmajor);
    std::vector<T> pfr, tpl, kr, sol;
    if (t->planck_frac) pfr = conv<T>(t->planck_frac, nk);
    if (t->totplnk) tpl = conv<T>(t->totplnk, size_t(t->nband) * t->nplanck_temp);
    a.add(pfr, &v.planck_frac);
    a.add(tpl, &v.totplnk);
    if (info.has_rayleigh) {
        const size_t nr = size_t(t->ntemp) * t->neta * t->ngpt;
        kr.resize(2 * nr);
        for (size_t i = 0; i < nr; ++i) { kr[i] = T(t->rayl_lower[i]); kr[nr + i] = T(t->rayl_upper[i]); }
    }
    a.add(kr, &v.krayl);
    std::vector<std::vector<T>> kmin(2);
    for (int atm = 0; atm < 2; ++atm) {
        const MinorHost& m = mh[atm];
        v.nminor[atm] = int(m.gstart.size());
        v.ncontrib[atm] = m.ncontrib;
        a.add(m.gstart, &v.minor_gstart[atm]);
        a.add(m.gend, &v.minor_gend[atm]);
        a.add(m.kstart, &v.minor_kstart[atm]);
        a.add(m.flav, &v.minor_flav[atm]);
        a.add(m.gas, &v.minor_gas[atm]);
        a.add(m.sgas, &v.minor_sgas[atm]);
        a.add(m.flags, &v.minor_flags[atm]);
        a.add(m.band_begin, &v.band_minor_begin[atm]);
        a.add(m.band_list, &v.band_minor_list[atm]);
        kmin[atm] = conv<T>(m.kminor.data(), m.kminor.size());
        a.add(kmin[atm], &v.kminor[atm]);
    }
    int in_band = 1, max_minor = 0;
    for (int atm = 0; atm < 2; ++atm) {
        for (size_t i = 0; i < mh[atm].gstart.size(); ++i)
            if (g2b[mh[atm].gstart[i]] != g2b[mh[atm].gend[i] - 1]) in_band = 0;
        for (int b = 0; b < t->nband; ++b)
            max_minor = std::max(max_minor, mh[atm].band_begin[b + 1] - mh[atm].band_begin[b]);
    }
    v.minor_in_band = in_band;
    v.max_band_minor = max_minor;
    // Scaling kinds (see KdistView): one per distinct (minor gas, scaling gas, complement
    // flag) among the density-scaled intervals and per minor gas among the others.
    std::vector<int> sid[2], sgas_k[2], ssg_k[2], sfl_k[2];
    v.max_nscal = 1;
    for (int atm = 0; atm < 2; ++atm) {
        const MinorHost& m = mh[atm];
        sid[atm].resize(m.gstart.size());
        for (size_t i = 0; i < m.gstart.size(); ++i) {
            const int fl = m.flags[i] & 3;
            const int gas = m.gas[i], sg = (fl & 1) ? m.sgas[i] : 0, f = (fl & 1) ? fl : 0;
            int found = -1;
            for (size_t q = 0; q < sgas_k[atm].size(); ++q)
                if (sgas_k[atm][q] == gas && ssg_k[atm][q] == sg && sfl_k[atm][q] == f) found = int(q);
            if (found < 0) {
                found = int(sgas_k[atm].size());
                sgas_k[atm].push_back(gas);
                ssg_k[atm].push_back(sg);
                sfl_k[atm].push_back(f);
            }
            sid[atm][i] = found;
        }
        v.nscal[atm] = int(sgas_k[atm].size());
        v.max_nscal = std::max(v.max_nscal, v.nscal[atm]);
        a.add(sgas_k[atm], &v.scal_gas[atm]);
        a.add(ssg_k[atm], &v.scal_sgas[atm]);
        a.add(sfl_k[atm], &v.scal_flags[atm]);
    }
    v.ngroups = (t->ngpt + 31) / 32;
    std::vector<int> gb0(v.ngroups);
    int max_gb = 0;
    for (int gg = 0; gg < v.ngroups; ++gg) {
        const int g0 = 32 * gg, g1 = std::min(t->ngpt, g0 + 32) - 1;
        gb0[gg] = g2b[g0];
        max_gb = std::max(max_gb, g2b[g1] - g2b[g0] + 1);
    }
    v.max_group_bands = max_gb;
    a.add(gb0, &v.group_band0);

    // Corner-packed tables for the fused FP32 kernels.
    v.max_minor_per_g = 0;
    v.minor_gx_stride = 0;
    std::vector<float4> km4, pf4;
    std::vector<float2> kn2[2], kr2;
    std::vector<int4> mg[2];
    std::vector<int> mgx[2];
    if (std::is_same<T, float>::value) {
        const int nt = t->ntemp, np = t->npres, np1 = t->npres + 1, ne = t->neta, ng = t->ngpt;
        auto pack4 = [&](const double* src, std::vector<float4>& dst) {
            dst.resize(size_t(nt) * np * (ne - 1) * ng);
            auto at = [&](int it, int ip, int ie, int ig) { return float(src[((size_t(it) * np1 + ip) * ne + ie) * ng + ig]); };
            for (int it = 0; it < nt; ++it)
                for (int ip = 0; ip < np; ++ip)
                    for (int ie = 0; ie < ne - 1; ++ie)
                        for (int ig = 0; ig < ng; ++ig)
                            dst[((size_t(it) * np + ip) * (ne - 1) + ie) * ng + ig] =
                                make_float4(at(it, ip, ie, ig), at(it, ip, ie + 1, ig), at(it, ip + 1, ie, ig),
                                            at(it, ip + 1, ie + 1, ig));
        };
        pack4(t->kmajor, km4);
        if (t->planck_frac) pack4(t->planck_frac, pf4);
        for (int atm = 0; atm < 2; ++atm) {
            const MinorHost& m = mh[atm];
            const int nc = std::max(m.ncontrib, 1);
            kn2[atm].resize(size_t(nt) * (ne - 1) * nc);
            for (int it = 0; it < nt; ++it)
                for (int ie = 0; ie < ne - 1; ++ie)
                    for (int c = 0; c < nc; ++c)
                        kn2[atm][(size_t(it) * (ne - 1) + ie) * nc + c] =
                            make_float2(float(m.kminor[(size_t(it) * ne + ie) * nc + c]),
                                        float(m.kminor[(size_t(it) * ne + ie + 1) * nc + c]));
        }
        // Intervals covering each g-point, as codes (contributor << kScalBits) | scaling kind,
        // in the file order of the intervals.
        std::vector<std::vector<int>> codes[2];
        for (int atm = 0; atm < 2; ++atm) {
            const MinorHost& m = mh[atm];
            codes[atm].assign(ng, {});
            for (size_t im = 0; im < m.gstart.size(); ++im)
                for (int g = m.gstart[im]; g < m.gend[im]; ++g)
                    codes[atm][g].push_back(((m.kstart[im] + g - m.gstart[im]) << kScalBits) | sid[atm][im]);
            for (int g = 0; g < ng; ++g) v.max_minor_per_g = std::max(v.max_minor_per_g, int(codes[atm][g].size()));
        }
        v.minor_gx_stride = std::max(v.max_minor_per_g - 3, 0);
        for (int atm = 0; atm < 2; ++atm) {
            mg[atm].assign(ng, make_int4(0, 0, 0, 0));
            if (v.minor_gx_stride) mgx[atm].assign(size_t(ng) * v.minor_gx_stride, 0);
            for (int g = 0; g < ng; ++g) {
                const std::vector<int>& c = codes[atm][g];
                int4& e = mg[atm][g];
                e.x = int(c.size());
                // unused slots repeat the first one, so a kernel may read every slot below a
                // warp-wide maximum count and discard the extra terms
                e.y = c.empty() ? 0 : c[0];
                e.z = c.size() > 1 ? c[1] : e.y;
                e.w = c.size() > 2 ? c[2] : e.y;
                for (size_t n = 3; n < c.size(); ++n) mgx[atm][size_t(g) * v.minor_gx_stride + n - 3] = c[n];
            }
        }
        if (info.has_rayleigh) {
            kr2.resize(size_t(2) * nt * (ne - 1) * ng);
            for (int atm = 0; atm < 2; ++atm) {
                const double* r = atm == 0 ? t->rayl_lower : t->rayl_upper;
                for (int it = 0; it < nt; ++it)
                    for (int ie = 0; ie < ne - 1; ++ie)
                        for (int ig = 0; ig < ng; ++ig)
                            kr2[((size_t(atm) * nt + it) * (ne - 1) + ie) * ng + ig] =
                                make_float2(float(r[(size_t(it) * ne + ie) * ng + ig]),
                                            float(r[(size_t(it) * ne + ie + 1) * ng + ig]));
            }
        }
    }
    a.add(km4, &v.kmaj4);
    a.add(pf4, &v.pfrac4);
    a.add(kn2[0], &v.kmin2[0]);
    a.add(kn2[1], &v.kmin2[1]);
    a.add(kr2, &v.krayl2);
    a.add(mg[0], &v.minor_g[0]);
    a.add(mg[1], &v.minor_g[1]);
    a.add(mgx[0], &v.minor_gx[0]);
    a.add(mgx[1], &v.minor_gx[1]);
    return a.upload(k->allocations);
}

}  // namespace

template <typename T>
int make_gas_set(const rrtmgp_b200_kdist_t* k, int ncol, int nlay,
                 const rrtmgp_b200_gas_conc* gases, int ngases, GasSet<T>& out)
{
    RB_CHECK_ARG(ngases >= 0 && (ngases == 0 || gases), "gas_concs: null gas list");
    for (size_t i = 0; i < k->gas_names.size(); ++i) {
        int found = -1;
        for (int j = 0; j < ngases; ++j)
            if (trim(gases[j].name) == k->gas_names[i]) found = j;
        if (found < 0)
            return fail(RRTMGP_B200_ERR_MISSING_GAS, "gas_concs: gas " + k->gas_names[i] + " not found");
        const auto& g = gases[found];
        RB_CHECK_ARG(g.vmr != nullptr, "gas_concs: null vmr for " + k->gas_names[i]);
        out.vmr[i] = static_cast<const T*>(g.vmr);
        if (g.dim1 == 1 && g.dim2 == 1) out.mode[i] = 0;
        else if (g.dim1 == 1 && g.dim2 == nlay) out.mode[i] = 1;
        else if (g.dim1 == ncol && g.dim2 == nlay) out.mode[i] = 2;
        else return fail(RRTMGP_B200_ERR_ARG, "gas_concs: bad dimensions for " + k->gas_names[i]);
    }
    for (size_t i = k->gas_names.size(); i < size_t(kMaxGases); ++i) { out.vmr[i] = nullptr; out.mode[i] = 0; }
    return RRTMGP_B200_OK;
}

template int make_gas_set<float>(const rrtmgp_b200_kdist_t*, int, int, const rrtmgp_b200_gas_conc*, int, GasSet<float>&);
template int make_gas_set<double>(const rrtmgp_b200_kdist_t*, int, int, const rrtmgp_b200_gas_conc*, int, GasSet<double>&);

int bands_create_impl(rrtmgp_b200_bands_t& b, int nband, const int* lims) { return bands_init(b, nband, lims); }
void bands_free_impl(rrtmgp_b200_bands_t& b) { bands_free(b); }

}  // namespace rrtmgp_b200

using namespace rrtmgp_b200;

extern "C" {

const char* rrtmgp_b200_last_error(void) { return g_last_error.c_str(); }
int rrtmgp_b200_abi_version(void) { return RRTMGP_B200_ABI_VERSION; }

int rrtmgp_b200_kdist_create(const rrtmgp_b200_kdist_tables* t, const char* const* available,
                             int n_available, rrtmgp_b200_kdist* out)
{
    RB_CHECK_ARG(t && out, "kdist_create: null argument");
    RB_CHECK_ARG(t->ngas > 0 && t->nband > 0 && t->ngpt > 0 && t->ntemp > 1 && t->npres > 1 && t->neta > 1,
                 "kdist_create: bad table dimensions");
    RB_CHECK_ARG(t->gas_names && t->key_species && t->band_lims_gpt && t->press_ref && t->temp_ref &&
                 t->vmr_ref && t->kmajor, "kdist_create: missing table");
    const bool lw = t->totplnk && t->planck_frac;
    const bool sw = t->solar_source_quiet && t->solar_source_facular && t->solar_source_sunspot;
    RB_CHECK_ARG(lw != sw, "kdist_create: need either (totplnk, planck_frac) or the solar source tables");
    RB_CHECK_ARG(t->nband <= kMaxBands, "kdist_create: too many bands");
    RB_CHECK_ARG(t->nband > 0 && t->ngpt > 0, "kdist_create: nband and ngpt must be > 0");
    for (int b = 0; b < t->nband; ++b) {
        RB_CHECK_ARG(t->band_lims_gpt[2 * b + 1] - t->band_lims_gpt[2 * b] + 1 <= kMaxBandGpt,
                     "kdist_create: more than 32 g-points in a band");
        // the kernels walk the bands in order and take g-point g + 1 to follow g
        RB_CHECK_ARG(t->band_lims_gpt[2 * b] == (b == 0 ? 1 : t->band_lims_gpt[2 * b - 1] + 1) &&
                     t->band_lims_gpt[2 * b + 1] >= t->band_lims_gpt[2 * b],
                     "kdist_create: band limits must cover g-points 1..ngpt in order, without gaps");
    }
    RB_CHECK_ARG(t->band_lims_gpt[2 * t->nband - 1] == t->ngpt,
                 "kdist_create: band limits must cover g-points 1..ngpt in order, without gaps");

    *out = nullptr;
    auto* k = new rrtmgp_b200_kdist_t();
    auto bail = [&](int st) {
        for (void* p : k->allocations) cudaFree(p);
        bands_free(k->bands);
        delete k;
        return st;
    };
    cudaGetDevice(&k->device);

    std::vector<std::string> names, avail;
    for (int i = 0; i < t->ngas; ++i) names.push_back(trim(t->gas_names[i]));
    for (int i = 0; i < n_available; ++i) avail.push_back(trim(available[i]));
    // Gases known to the k-distribution and present in the model (init_abs_coeffs :571-584).
    for (auto& s : names)
        if (find1(avail, s) > 0) k->gas_names.push_back(s);
    const int ngas = int(k->gas_names.size());
    if (ngas > kMaxGases) return bail(fail(RRTMGP_B200_ERR_UNSUPPORTED, "kdist_create: too many gases"));
    if (find1(k->gas_names, "h2o") < 0)
        return bail(fail(RRTMGP_B200_ERR_MISSING_GAS, "idx_h2o cannot be found"));

    // vmr_ref reduced to [ntemp][ngas+1][2], index 0 = dry air (:589-605).
    std::vector<double> vmr((size_t)t->ntemp * (ngas + 1) * 2);
    for (int it = 0; it < t->ntemp; ++it)
        for (int i = 0; i <= ngas; ++i) {
            const int src = i == 0 ? 0 : find1(names, k->gas_names[i - 1]);
            for (int a = 0; a < 2; ++a)
                vmr[((size_t)it * (ngas + 1) + i) * 2 + a] = t->vmr_ref[((size_t)it * (t->ngas + 1) + src) * 2 + a];
        }

    // Key species reduction and presence check (create_key_species_reduce :198-245).
    std::vector<int> ks(4 * t->nband);
    for (int b = 0; b < t->nband; ++b)
        for (int a = 0; a < 2; ++a)
            for (int p = 0; p < 2; ++p) {
                const int v = t->key_species[(b * 2 + a) * 2 + p];
                int r = 0;
                if (v != 0) {
                    RB_CHECK_ARG(v >= 1 && v <= t->ngas, "kdist_create: key species index out of range");
                    r = find1(k->gas_names, names[v - 1]);
                    if (r < 0)
                        return bail(fail(RRTMGP_B200_ERR_MISSING_GAS,
                                         "Gas optics: required gas " + names[v - 1] + " is missing"));
                }
                ks[(b * 2 + a) * 2 + p] = r;
            }
    // Flavors: unique (gas1, gas2) pairs in band-major order, (0,0) -> (2,2) (create_flavor
    // :247-313); per-band flavor per atmosphere (create_gpoint_flavor :331-363).
    std::vector<std::pair<int, int>> flav;
    std::vector<int> band_flav(2 * t->nband);
    for (int b = 0; b < t->nband; ++b)
        for (int a = 0; a < 2; ++a) {
            std::pair<int, int> pr{ks[(b * 2 + a) * 2], ks[(b * 2 + a) * 2 + 1]};
            if (pr.first == 0 && pr.second == 0) pr = {2, 2};
            auto it = std::find(flav.begin(), flav.end(), pr);
            if (it == flav.end()) { flav.push_back(pr); it = flav.end() - 1; }
            band_flav[2 * b + a] = int(it - flav.begin());
        }
    std::vector<int> flavor;
    for (auto& p : flav) {
        if (p.first > ngas || p.second > ngas)
            return bail(fail(RRTMGP_B200_ERR_MISSING_GAS, "kdist_create: flavor gas index beyond reduced gas list"));
        flavor.push_back(p.first);
        flavor.push_back(p.second);
    }

    // Minor absorbers (reduce_minor_arrays :53-162, create_idx_minor :164-196).
    std::vector<std::string> ident, gas_minor;
    for (int i = 0; i < t->nminor_absorber; ++i) {
        ident.push_back(trim(t->identifier_minor[i]));
        gas_minor.push_back(trim(t->gas_minor[i]));
    }
    MinorHost mh[2];
    std::vector<int> g2b(t->ngpt, 0);
    for (int b = 0; b < t->nband; ++b)
        for (int g = t->band_lims_gpt[2 * b] - 1; g < t->band_lims_gpt[2 * b + 1]; ++g) g2b[g] = b;
    for (int atm = 0; atm < 2; ++atm) {
        const int nint = atm == 0 ? t->nint_lower : t->nint_upper;
        const int ncontrib = atm == 0 ? t->ncontrib_lower : t->ncontrib_upper;
        const char* const* mg = atm == 0 ? t->minor_gases_lower : t->minor_gases_upper;
        const int* lims = atm == 0 ? t->minor_limits_gpt_lower : t->minor_limits_gpt_upper;
        const int* dens = atm == 0 ? t->minor_scales_with_density_lower : t->minor_scales_with_density_upper;
        const char* const* sg = atm == 0 ? t->scaling_gas_lower : t->scaling_gas_upper;
        const int* comp = atm == 0 ? t->scale_by_complement_lower : t->scale_by_complement_upper;
        const int* kst = atm == 0 ? t->kminor_start_lower : t->kminor_start_upper;
        const double* kmn = atm == 0 ? t->kminor_lower : t->kminor_upper;
        MinorHost& m = mh[atm];
        int tot = 0;
        std::vector<int> present(nint, 0);
        for (int i = 0; i < nint; ++i) {
            const int im = find1(ident, trim(mg[i]));
            present[i] = im > 0 && find1(avail, gas_minor[im - 1]) > 0;
            if (present[i]) tot += lims[2 * i + 1] - lims[2 * i] + 1;
        }
        m.ncontrib = tot;
        m.kminor.assign((size_t)t->ntemp * t->neta * std::max(tot, 1), 0.);
        int off = 0;
        for (int i = 0; i < nint; ++i) {
            if (!present[i]) continue;
            const int ng = lims[2 * i + 1] - lims[2 * i] + 1;
            RB_CHECK_ARG(lims[2 * i] >= 1 && lims[2 * i + 1] <= t->ngpt, "kdist_create: minor limits out of range");
            RB_CHECK_ARG(kst[i] >= 1 && kst[i] - 1 + ng <= ncontrib, "kdist_create: kminor_start out of range");
            const int im = find1(ident, trim(mg[i]));
            const int gi = find1(k->gas_names, gas_minor[im - 1]);
            if (gi < 0)
                return bail(fail(RRTMGP_B200_ERR_MISSING_GAS,
                                 "kdist_create: minor gas " + gas_minor[im - 1] + " not in k-distribution gases"));
            m.gstart.push_back(lims[2 * i] - 1);
            m.gend.push_back(lims[2 * i + 1]);
            m.kstart.push_back(off);
            m.flav.push_back(band_flav[2 * g2b[lims[2 * i] - 1] + atm]);
            m.gas.push_back(gi);
            m.sgas.push_back(find1(k->gas_names, trim(sg[i])));
            m.flags.push_back((dens[i] ? 1 : 0) | (comp[i] ? 2 : 0));
            for (int it = 0; it < t->ntemp; ++it)
                for (int ie = 0; ie < t->neta; ++ie)
                    for (int j = 0; j < ng; ++j)
                        m.kminor[((size_t)it * t->neta + ie) * std::max(tot, 1) + off + j] =
                            kmn[((size_t)it * t->neta + ie) * ncontrib + (kst[i] - 1 + j)];
            off += ng;
        }
        // Intervals overlapping each band.
        m.band_begin.assign(t->nband + 1, 0);
        for (int b = 0; b < t->nband; ++b) {
            m.band_begin[b] = int(m.band_list.size());
            const int b0 = t->band_lims_gpt[2 * b] - 1, b1 = t->band_lims_gpt[2 * b + 1];
            for (size_t i = 0; i < m.gstart.size(); ++i)
                if (m.gstart[i] < b1 && m.gend[i] > b0) m.band_list.push_back(int(i));
        }
        m.band_begin[t->nband] = int(m.band_list.size());
    }

    auto& info = k->info;
    info.ngas = ngas;
    info.nflav = int(flav.size());
    info.nband = t->nband;
    info.ngpt = t->ngpt;
    info.ntemp = t->ntemp;
    info.npres = t->npres;
    info.neta = t->neta;
    info.nplanck_temp = lw ? t->nplanck_temp : 0;
    info.nminor_lower = int(mh[0].gstart.size());
    info.nminor_upper = int(mh[1].gstart.size());
    info.is_longwave = lw ? 1 : 0;
    info.has_rayleigh = (t->rayl_lower && t->rayl_upper) ? 1 : 0;
    info.press_ref_min = t->press_ref[t->npres - 1];
    info.press_ref_max = t->press_ref[0];
    info.temp_ref_min = t->temp_ref[0];
    info.temp_ref_max = t->temp_ref[t->ntemp - 1];

    int st = fill_view<float>(k, k->v32, t, vmr, flavor, band_flav, mh);
    if (st == RRTMGP_B200_OK) st = fill_view<double>(k, k->v64, t, vmr, flavor, band_flav, mh);
    if (st == RRTMGP_B200_OK) st = bands_init(k->bands, t->nband, t->band_lims_gpt);
    if (st != RRTMGP_B200_OK) return bail(st);
    k->bands.owned_by_parent = true;

    if (cudaMalloc(&k->d_flags, sizeof(int)) != cudaSuccess)
        return bail(fail(RRTMGP_B200_ERR_ALLOC, "cudaMalloc of the flag word failed"));
    k->allocations.push_back(k->d_flags);
    if (sw) {
        k->solar_quiet.assign(t->solar_source_quiet, t->solar_source_quiet + t->ngpt);
        k->solar_fac.assign(t->solar_source_facular, t->solar_source_facular + t->ngpt);
        k->solar_spot.assign(t->solar_source_sunspot, t->solar_source_sunspot + t->ngpt);
        if (cudaMalloc(&k->d_solar32, t->ngpt * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&k->d_solar64, t->ngpt * sizeof(double)) != cudaSuccess)
            return bail(fail(RRTMGP_B200_ERR_ALLOC, "cudaMalloc of solar source failed"));
        k->allocations.push_back(k->d_solar32);
        k->allocations.push_back(k->d_solar64);
        *out = k;
        st = rrtmgp_b200_kdist_set_solar_variability(k, t->mg_default, t->sb_default);
        if (st != RRTMGP_B200_OK) { *out = nullptr; return bail(st); }
    }
    k->v32.solar_source = k->d_solar32;
    k->v64.solar_source = k->d_solar64;
    *out = k;
    return RRTMGP_B200_OK;
}

void rrtmgp_b200_kdist_destroy(rrtmgp_b200_kdist k)
{
    if (!k) return;
    for (void* p : k->allocations) cudaFree(p);
    bands_free(k->bands);
    delete k;
}

int rrtmgp_b200_kdist_get_info(rrtmgp_b200_kdist k, rrtmgp_b200_kdist_info* info)
{
    RB_CHECK_ARG(k && info, "kdist_get_info: null argument");
    *info = k->info;
    double tsi = 0.;
    for (double s : k->solar_source) tsi += s;
    info->tsi = tsi;
    return RRTMGP_B200_OK;
}

int rrtmgp_b200_kdist_gas_name(rrtmgp_b200_kdist k, int i, char* buf, int buflen)
{
    RB_CHECK_ARG(k && buf && buflen > 0, "kdist_gas_name: null argument");
    RB_CHECK_ARG(i >= 0 && i < int(k->gas_names.size()), "kdist_gas_name: index out of range");
    std::strncpy(buf, k->gas_names[i].c_str(), buflen - 1);
    buf[buflen - 1] = '\0';
    return RRTMGP_B200_OK;
}

rrtmgp_b200_bands rrtmgp_b200_kdist_bands(rrtmgp_b200_kdist k) { return k ? &k->bands : nullptr; }

// set_solar_variability (src/Gas_optics_rrtmgp.cpp:745-760).
int rrtmgp_b200_kdist_set_solar_variability(rrtmgp_b200_kdist k, double mg_index, double sb_index)
{
    RB_CHECK_ARG(k, "set_solar_variability: null kdist");
    if (k->solar_quiet.empty()) return fail(RRTMGP_B200_ERR_UNSUPPORTED, "set_solar_variability: longwave k-distribution");
    const double a_offset = 0.1495954, b_offset = 0.00066696;
    const int n = int(k->solar_quiet.size());
    k->solar_source.resize(n);
    std::vector<float> s32(n);
    for (int g = 0; g < n; ++g) {
        k->solar_source[g] = k->solar_quiet[g] + (mg_index - a_offset) * k->solar_fac[g] +
                             (sb_index - b_offset) * k->solar_spot[g];
        s32[g] = float(k->solar_source[g]);
    }
    RB_CUDA(cudaMemcpy(k->d_solar32, s32.data(), n * sizeof(float), cudaMemcpyHostToDevice), "solar upload");
    RB_CUDA(cudaMemcpy(k->d_solar64, k->solar_source.data(), n * sizeof(double), cudaMemcpyHostToDevice), "solar upload");
    return RRTMGP_B200_OK;
}

int rrtmgp_b200_kdist_solar_source(rrtmgp_b200_kdist k, double* out)
{
    RB_CHECK_ARG(k && out, "kdist_solar_source: null argument");
    if (k->solar_source.empty()) return fail(RRTMGP_B200_ERR_UNSUPPORTED, "kdist_solar_source: longwave k-distribution");
    std::copy(k->solar_source.begin(), k->solar_source.end(), out);
    return RRTMGP_B200_OK;
}

int rrtmgp_b200_bands_create(int nband, const int* lims, rrtmgp_b200_bands* out)
{
    RB_CHECK_ARG(out, "bands_create: null out");
    auto* b = new rrtmgp_b200_bands_t();
    const int st = bands_init(*b, nband, lims);
    if (st != RRTMGP_B200_OK) { bands_free(*b); delete b; *out = nullptr; return st; }
    *out = b;
    return RRTMGP_B200_OK;
}

void rrtmgp_b200_bands_destroy(rrtmgp_b200_bands b)
{
    if (!b || b->owned_by_parent) return;
    bands_free(*b);
    delete b;
}

int rrtmgp_b200_bands_get(rrtmgp_b200_bands b, int* nband, int* ngpt)
{
    RB_CHECK_ARG(b, "bands_get: null bands");
    if (nband) *nband = b->nband;
    if (ngpt) *ngpt = b->ngpt;
    return RRTMGP_B200_OK;
}

// Cloud_optics_gpu ctor (src_cuda/Cloud_optics.cu:130-179), ice roughness icergh = 2.
int rrtmgp_b200_cloud_create(const rrtmgp_b200_cloud_tables* t, rrtmgp_b200_cloud* out)
{
    RB_CHECK_ARG(t && out, "cloud_create: null argument");
    RB_CHECK_ARG(t->nband > 0 && t->nsize_liq > 1 && t->nsize_ice > 1 && t->nrghice >= 2,
                 "cloud_create: bad LUT dimensions");
    RB_CHECK_ARG(t->lut_extliq && t->lut_ssaliq && t->lut_asyliq && t->lut_extice && t->lut_ssaice &&
                 t->lut_asyice, "cloud_create: missing LUT");
    auto* c = new rrtmgp_b200_cloud_t();
    c->nband = t->nband;
    c->nsize_liq = t->nsize_liq;
    c->nsize_ice = t->nsize_ice;
    c->radliq_lwr = t->radliq_lwr;
    c->radice_lwr = t->radice_lwr;
    c->liq_step = (t->radliq_upr - t->radliq_lwr) / (t->nsize_liq - 1.);
    c->ice_step = (t->radice_upr - t->radice_lwr) / (t->nsize_ice - 1.);
    const size_t nl = size_t(t->nband) * t->nsize_liq, ni = size_t(t->nband) * t->nsize_ice;
    const int icergh = 2;
    std::vector<double> all;
    for (const double* p : {t->lut_extliq, t->lut_ssaliq, t->lut_asyliq}) all.insert(all.end(), p, p + nl);
    for (const double* p : {t->lut_extice, t->lut_ssaice, t->lut_asyice})
        all.insert(all.end(), p + (icergh - 1) * ni, p + icergh * ni);
    std::vector<float> all32(all.begin(), all.end());
    if (cudaMalloc(&c->lut32, all32.size() * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&c->lut64, all.size() * sizeof(double)) != cudaSuccess) {
        if (c->lut32) cudaFree(c->lut32);
        delete c;
        return fail(RRTMGP_B200_ERR_ALLOC, "cloud_create: cudaMalloc failed");
    }
    RB_CUDA(cudaMemcpy(c->lut32, all32.data(), all32.size() * sizeof(float), cudaMemcpyHostToDevice), "cloud upload");
    RB_CUDA(cudaMemcpy(c->lut64, all.data(), all.size() * sizeof(double), cudaMemcpyHostToDevice), "cloud upload");
    std::vector<int> lims(2 * t->nband);
    for (int b = 0; b < t->nband; ++b) { lims[2 * b] = b + 1; lims[2 * b + 1] = b + 1; }
    const int st = bands_init(c->bands, t->nband, lims.data());
    if (st != RRTMGP_B200_OK) { rrtmgp_b200_cloud_destroy(c); return st; }
    c->bands.owned_by_parent = true;
    *out = c;
    return RRTMGP_B200_OK;
}

void rrtmgp_b200_cloud_destroy(rrtmgp_b200_cloud c)
{
    if (!c) return;
    if (c->lut32) cudaFree(c->lut32);
    if (c->lut64) cudaFree(c->lut64);
    bands_free(c->bands);
    delete c;
}

}  // extern "C"
