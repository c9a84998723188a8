// Longwave source functions on the GPU: Source_func_lw_gpu of the reference
// (include/Source_functions.h:72-99).  Layer and level sources (ncol, nlay, ngpt), surface
// source and its temperature Jacobian (ncol, ngpt).
#ifndef RRTMGP_B200_CPP_SOURCE_FUNCTIONS_H
#define RRTMGP_B200_CPP_SOURCE_FUNCTIONS_H

#include "Optical_props.h"

class Source_func_lw_gpu : public Optical_props_gpu
{
  public:
    Source_func_lw_gpu(const int n_col, const int n_lay, const Optical_props_gpu& optical_props)
        : Optical_props_gpu(optical_props),
          sfc_source({n_col, optical_props.get_ngpt()}),
          sfc_source_jac({n_col, optical_props.get_ngpt()}),
          lay_source({n_col, n_lay, optical_props.get_ngpt()}),
          lev_source_inc({n_col, n_lay, optical_props.get_ngpt()}),
          lev_source_dec({n_col, n_lay, optical_props.get_ngpt()})
    {}

    Array_gpu<Float, 2>& get_sfc_source() { return sfc_source; }
    Array_gpu<Float, 2>& get_sfc_source_jac() { return sfc_source_jac; }
    Array_gpu<Float, 3>& get_lay_source() { return lay_source; }
    Array_gpu<Float, 3>& get_lev_source_inc() { return lev_source_inc; }
    Array_gpu<Float, 3>& get_lev_source_dec() { return lev_source_dec; }

    const Array_gpu<Float, 2>& get_sfc_source() const { return sfc_source; }
    const Array_gpu<Float, 2>& get_sfc_source_jac() const { return sfc_source_jac; }
    const Array_gpu<Float, 3>& get_lay_source() const { return lay_source; }
    const Array_gpu<Float, 3>& get_lev_source_inc() const { return lev_source_inc; }
    const Array_gpu<Float, 3>& get_lev_source_dec() const { return lev_source_dec; }

  private:
    Array_gpu<Float, 2> sfc_source;
    Array_gpu<Float, 2> sfc_source_jac;
    Array_gpu<Float, 3> lay_source;
    Array_gpu<Float, 3> lev_source_inc;
    Array_gpu<Float, 3> lev_source_dec;
};

#endif
