// Reduction of g-point fluxes on the GPU: Fluxes_gpu, Fluxes_broadband_gpu and
// Fluxes_byband_gpu of the reference (include/Fluxes.h:126-220).  Broadband sums over all
// g-points with compensated summation; net = dn - up.  Output arrays (ncol, nlev) and, by
// band, (ncol, nlev, nband).
#ifndef RRTMGP_B200_CPP_FLUXES_H
#define RRTMGP_B200_CPP_FLUXES_H

#include <memory>
#include <stdexcept>

#include "Optical_props.h"

class Fluxes_gpu
{
  public:
    virtual ~Fluxes_gpu() {}
    virtual void reduce(const Array_gpu<Float, 3>& gpt_flux_up, const Array_gpu<Float, 3>& gpt_flux_dn,
                        const std::unique_ptr<Optical_props_arry_gpu>& optical_props, const Bool top_at_1) = 0;
    virtual void reduce(const Array_gpu<Float, 3>& gpt_flux_up, const Array_gpu<Float, 3>& gpt_flux_dn,
                        const Array_gpu<Float, 3>& gpt_flux_dn_dir,
                        const std::unique_ptr<Optical_props_arry_gpu>& optical_props, const Bool top_at_1) = 0;
};

class Fluxes_broadband_gpu : public Fluxes_gpu
{
  public:
    Fluxes_broadband_gpu(const int ncol, const int nlev)
        : flux_up({ncol, nlev}), flux_dn({ncol, nlev}), flux_dn_dir({ncol, nlev}), flux_net({ncol, nlev})
    {}
    virtual ~Fluxes_broadband_gpu() {}

    virtual void reduce(const Array_gpu<Float, 3>& gpt_flux_up, const Array_gpu<Float, 3>& gpt_flux_dn,
                        const std::unique_ptr<Optical_props_arry_gpu>&, const Bool)
    {
        rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::broadband(gpt_flux_up.dim(1), gpt_flux_up.dim(2), gpt_flux_up.dim(3),
                                                          gpt_flux_up.ptr(), gpt_flux_dn.ptr(), nullptr,
                                                          flux_up.ptr(), flux_dn.ptr(), nullptr, flux_net.ptr()));
    }
    virtual void reduce(const Array_gpu<Float, 3>& gpt_flux_up, const Array_gpu<Float, 3>& gpt_flux_dn,
                        const Array_gpu<Float, 3>& gpt_flux_dn_dir,
                        const std::unique_ptr<Optical_props_arry_gpu>&, const Bool)
    {
        rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::broadband(gpt_flux_up.dim(1), gpt_flux_up.dim(2), gpt_flux_up.dim(3),
                                                          gpt_flux_up.ptr(), gpt_flux_dn.ptr(), gpt_flux_dn_dir.ptr(),
                                                          flux_up.ptr(), flux_dn.ptr(), flux_dn_dir.ptr(),
                                                          flux_net.ptr()));
    }

    Array_gpu<Float, 2>& get_flux_up() { return flux_up; }
    Array_gpu<Float, 2>& get_flux_dn() { return flux_dn; }
    Array_gpu<Float, 2>& get_flux_dn_dir() { return flux_dn_dir; }
    Array_gpu<Float, 2>& get_flux_net() { return flux_net; }

    virtual Array_gpu<Float, 3>& get_bnd_flux_up() { throw std::runtime_error("Band fluxes are not available"); }
    virtual Array_gpu<Float, 3>& get_bnd_flux_dn() { throw std::runtime_error("Band fluxes are not available"); }
    virtual Array_gpu<Float, 3>& get_bnd_flux_dn_dir() { throw std::runtime_error("Band fluxes are not available"); }
    virtual Array_gpu<Float, 3>& get_bnd_flux_net() { throw std::runtime_error("Band fluxes are not available"); }

  private:
    Array_gpu<Float, 2> flux_up;
    Array_gpu<Float, 2> flux_dn;
    Array_gpu<Float, 2> flux_dn_dir;
    Array_gpu<Float, 2> flux_net;
};

class Fluxes_byband_gpu : public Fluxes_broadband_gpu
{
  public:
    Fluxes_byband_gpu(const int ncol, const int nlev, const int nbnd)
        : Fluxes_broadband_gpu(ncol, nlev), bnd_flux_up({ncol, nlev, nbnd}), bnd_flux_dn({ncol, nlev, nbnd}),
          bnd_flux_dn_dir({ncol, nlev, nbnd}), bnd_flux_net({ncol, nlev, nbnd})
    {}
    virtual ~Fluxes_byband_gpu() {}

    virtual void reduce(const Array_gpu<Float, 3>& gpt_flux_up, const Array_gpu<Float, 3>& gpt_flux_dn,
                        const std::unique_ptr<Optical_props_arry_gpu>& optical_props, const Bool top_at_1)
    {
        Fluxes_broadband_gpu::reduce(gpt_flux_up, gpt_flux_dn, optical_props, top_at_1);
        rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::byband(optical_props->bands_handle(), gpt_flux_up.dim(1),
                                                       gpt_flux_up.dim(2), gpt_flux_up.ptr(), gpt_flux_dn.ptr(),
                                                       nullptr, bnd_flux_up.ptr(), bnd_flux_dn.ptr(), nullptr,
                                                       bnd_flux_net.ptr()));
    }
    virtual void reduce(const Array_gpu<Float, 3>& gpt_flux_up, const Array_gpu<Float, 3>& gpt_flux_dn,
                        const Array_gpu<Float, 3>& gpt_flux_dn_dir,
                        const std::unique_ptr<Optical_props_arry_gpu>& optical_props, const Bool top_at_1)
    {
        Fluxes_broadband_gpu::reduce(gpt_flux_up, gpt_flux_dn, gpt_flux_dn_dir, optical_props, top_at_1);
        rrtmgp_b200_cpp::check(rrtmgp_b200_cpp::byband(optical_props->bands_handle(), gpt_flux_up.dim(1),
                                                       gpt_flux_up.dim(2), gpt_flux_up.ptr(), gpt_flux_dn.ptr(),
                                                       gpt_flux_dn_dir.ptr(), bnd_flux_up.ptr(), bnd_flux_dn.ptr(),
                                                       bnd_flux_dn_dir.ptr(), bnd_flux_net.ptr()));
    }

    Array_gpu<Float, 3>& get_bnd_flux_up() { return bnd_flux_up; }
    Array_gpu<Float, 3>& get_bnd_flux_dn() { return bnd_flux_dn; }
    Array_gpu<Float, 3>& get_bnd_flux_dn_dir() { return bnd_flux_dn_dir; }
    Array_gpu<Float, 3>& get_bnd_flux_net() { return bnd_flux_net; }

  private:
    Array_gpu<Float, 3> bnd_flux_up;
    Array_gpu<Float, 3> bnd_flux_dn;
    Array_gpu<Float, 3> bnd_flux_dn_dir;
    Array_gpu<Float, 3> bnd_flux_net;
};

#endif
