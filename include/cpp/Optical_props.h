// Spectral discretisation and optical-property containers on the GPU, with the reference's
// interface (include/Optical_props.h:169-293): Optical_props_gpu (band limits in wavenumber
// and g-points), Optical_props_arry_gpu with its 1scl (tau) and 2str (tau, ssa, g) forms,
// delta_scale and add_to.  Arrays are (ncol, nlay, ngpt), column fastest.
#ifndef RRTMGP_B200_CPP_OPTICAL_PROPS_H
#define RRTMGP_B200_CPP_OPTICAL_PROPS_H

#include <memory>
#include <stdexcept>

#include "Array.h"

class Optical_props_1scl_gpu;
class Optical_props_2str_gpu;
void add_to(Optical_props_1scl_gpu& op_inout, const Optical_props_1scl_gpu& op_in);
void add_to(Optical_props_2str_gpu& op_inout, const Optical_props_2str_gpu& op_in);

class Optical_props_gpu
{
  public:
    Optical_props_gpu(const Array<Float, 2>& band_lims_wvn, const Array<int, 2>& band_lims_gpt)
    {
        init(band_lims_wvn, band_lims_gpt);
    }
    // One g-point per band.
    explicit Optical_props_gpu(const Array<Float, 2>& band_lims_wvn)
    {
        const int nband = band_lims_wvn.dim(2);
        Array<int, 2> lims({2, nband});
        for (int b = 1; b <= nband; ++b) {
            lims({1, b}) = b;
            lims({2, b}) = b;
        }
        init(band_lims_wvn, lims);
    }
    virtual ~Optical_props_gpu() {}
    Optical_props_gpu(const Optical_props_gpu&) = default;

    Array<int, 1> get_gpoint_bands() const { return gpt2band; }
    const Array_gpu<int, 1>& get_gpoint_bands_gpu() const { return gpt2band_gpu; }
    const Array_gpu<int, 2>& get_band_lims_gpoint_gpu() const { return band2gpt_gpu; }
    int get_nband() const { return band2gpt.dim(2); }
    int get_ngpt() const { return band2gpt.max(); }
    const Array<int, 2>& get_band_lims_gpoint() const { return band2gpt; }
    const Array<Float, 2>& get_band_lims_wavenumber() const { return band_lims_wvn; }

    // C-ABI band handle shared by all copies of this discretisation.
    rrtmgp_b200_bands bands_handle() const { return bands.get(); }

  private:
    void init(const Array<Float, 2>& wvn, const Array<int, 2>& gpt)
    {
        band_lims_wvn = wvn;
        band2gpt = gpt;
        const int nband = gpt.dim(2);
        const int ngpt = gpt.max();
        gpt2band = Array<int, 1>({ngpt});
        for (int b = 1; b <= nband; ++b)
            for (int g = gpt({1, b}); g <= gpt({2, b}); ++g) gpt2band({g}) = b;
        band2gpt_gpu = Array_gpu<int, 2>(band2gpt);
        gpt2band_gpu = Array_gpu<int, 1>(gpt2band);
        std::vector<int> lims(gpt.v());   // (2, nband) Fortran = (nband, 2) C order, 1-based
        rrtmgp_b200_bands h = nullptr;
        rrtmgp_b200_cpp::check(rrtmgp_b200_bands_create(nband, lims.data(), &h));
        bands = std::shared_ptr<rrtmgp_b200_bands_t>(h, [](rrtmgp_b200_bands p) { rrtmgp_b200_bands_destroy(p); });
    }

    Array<int, 2> band2gpt;
    Array_gpu<int, 2> band2gpt_gpu;
    Array<int, 1> gpt2band;
    Array_gpu<int, 1> gpt2band_gpu;
    Array<Float, 2> band_lims_wvn;
    std::shared_ptr<rrtmgp_b200_bands_t> bands;
};

class Optical_props_arry_gpu : public Optical_props_gpu
{
  public:
    explicit Optical_props_arry_gpu(const Optical_props_gpu& op) : Optical_props_gpu(op) {}
    virtual ~Optical_props_arry_gpu() {}

    virtual Array_gpu<Float, 3>& get_tau() = 0;
    virtual Array_gpu<Float, 3>& get_ssa() = 0;
    virtual Array_gpu<Float, 3>& get_g() = 0;
    virtual const Array_gpu<Float, 3>& get_tau() const = 0;
    virtual const Array_gpu<Float, 3>& get_ssa() const = 0;
    virtual const Array_gpu<Float, 3>& get_g() const = 0;

    virtual void delta_scale(const Array_gpu<Float, 3>& forward_frac = Array_gpu<Float, 3>()) = 0;

    virtual int get_ncol() const = 0;
    virtual int get_nlay() const = 0;
};

class Optical_props_1scl_gpu : public Optical_props_arry_gpu
{
  public:
    Optical_props_1scl_gpu(const int ncol, const int nlay, const Optical_props_gpu& op)
        : Optical_props_arry_gpu(op), tau({ncol, nlay, op.get_ngpt()})
    {}

    int get_ncol() const { return tau.dim(1); }
    int get_nlay() const { return tau.dim(2); }

    Array_gpu<Float, 3>& get_tau() { return tau; }
    Array_gpu<Float, 3>& get_ssa() { throw std::runtime_error("ssa is not available in this class"); }
    Array_gpu<Float, 3>& get_g() { throw std::runtime_error("g is not available in this class"); }
    const Array_gpu<Float, 3>& get_tau() const { return tau; }
    const Array_gpu<Float, 3>& get_ssa() const { throw std::runtime_error("ssa is not available in this class"); }
    const Array_gpu<Float, 3>& get_g() const { throw std::runtime_error("g is not available in this class"); }

    void delta_scale(const Array_gpu<Float, 3>& = Array_gpu<Float, 3>()) {}

  private:
    Array_gpu<Float, 3> tau;
};

class Optical_props_2str_gpu : public Optical_props_arry_gpu
{
  public:
    Optical_props_2str_gpu(const int ncol, const int nlay, const Optical_props_gpu& op)
        : Optical_props_arry_gpu(op), tau({ncol, nlay, op.get_ngpt()}), ssa({ncol, nlay, op.get_ngpt()}),
          g({ncol, nlay, op.get_ngpt()})
    {}

    int get_ncol() const { return tau.dim(1); }
    int get_nlay() const { return tau.dim(2); }

    Array_gpu<Float, 3>& get_tau() { return tau; }
    Array_gpu<Float, 3>& get_ssa() { return ssa; }
    Array_gpu<Float, 3>& get_g() { return g; }
    const Array_gpu<Float, 3>& get_tau() const { return tau; }
    const Array_gpu<Float, 3>& get_ssa() const { return ssa; }
    const Array_gpu<Float, 3>& get_g() const { return g; }

    // Delta scaling with forward fraction f = g^2 (the reference's default); an explicit
    // forward_frac array is not supported, as in the reference GPU class.
    void delta_scale(const Array_gpu<Float, 3>& forward_frac = Array_gpu<Float, 3>())
    {
        if (forward_frac.size() != 0)
            throw std::runtime_error("delta_scale: an explicit forward fraction is not supported");
        rrtmgp_b200_cpp::check(
            rrtmgp_b200_cpp::delta_scale(get_ncol(), get_nlay(), tau.dim(3), tau.ptr(), ssa.ptr(), g.ptr()));
    }

  private:
    Array_gpu<Float, 3> tau;
    Array_gpu<Float, 3> ssa;
    Array_gpu<Float, 3> g;
    friend void add_to(Optical_props_2str_gpu& op_inout, const Optical_props_2str_gpu& op_in);
};

// Increment op_inout by op_in: g-point by g-point when both have the same g-points, by band
// when op_in has one value per band of op_inout (src_cuda/Optical_props.cu:93-145).
inline void add_to(Optical_props_1scl_gpu& op_inout, const Optical_props_1scl_gpu& op_in)
{
    if (op_inout.get_ncol() != op_in.get_ncol() || op_inout.get_nlay() != op_in.get_nlay())
        throw std::runtime_error("add_to: ncol and nlay must match");
    rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::add_to_1scl(op_inout.bands_handle(), op_inout.get_ncol(),
                                                         op_inout.get_nlay(), op_inout.get_tau().ptr(),
                                                         op_in.get_tau().ptr(), op_in.get_tau().dim(3)));
}

inline void add_to(Optical_props_2str_gpu& op_inout, const Optical_props_2str_gpu& op_in)
{
    if (op_inout.get_ncol() != op_in.get_ncol() || op_inout.get_nlay() != op_in.get_nlay())
        throw std::runtime_error("add_to: ncol and nlay must match");
    rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::add_to_2str(
        op_inout.bands_handle(), op_inout.get_ncol(), op_inout.get_nlay(), op_inout.tau.ptr(), op_inout.ssa.ptr(),
        op_inout.g.ptr(), op_in.tau.ptr(), op_in.ssa.ptr(), op_in.g.ptr(), op_in.tau.dim(3)));
}

#endif
