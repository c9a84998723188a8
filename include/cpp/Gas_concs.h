// Gas volume mixing ratios by name: Gas_concs (host) and Gas_concs_gpu (device), the
// reference's include/Gas_concs.h:40-91 interface.  A gas is a scalar (stored with dims
// {1, 1}), a profile (Array<Float,1> of nlay, stored {1, nlay}) or a field {ncol, nlay}.
#ifndef RRTMGP_B200_CPP_GAS_CONCS_H
#define RRTMGP_B200_CPP_GAS_CONCS_H

#include <map>
#include <string>
#include <vector>

#include "Array.h"

class Gas_concs_gpu;

class Gas_concs
{
  public:
    Gas_concs() = default;

    void set_vmr(const std::string& name, const Float data)
    {
        gas_concs_map[name] = Array<Float, 2>(std::vector<Float>{data}, {1, 1});
    }
    void set_vmr(const std::string& name, const Array<Float, 1>& data)
    {
        gas_concs_map[name] = Array<Float, 2>(data.v(), {1, data.dim(1)});
    }
    void set_vmr(const std::string& name, const Array<Float, 2>& data) { gas_concs_map[name] = data; }

    const Array<Float, 2>& get_vmr(const std::string& name) const
    {
        auto it = gas_concs_map.find(name);
        if (it == gas_concs_map.end()) throw std::runtime_error("Gas " + name + " is not available");
        return it->second;
    }
    Bool exists(const std::string& name) const { return gas_concs_map.count(name) != 0; }

  private:
    std::map<std::string, Array<Float, 2>> gas_concs_map;
    friend class Gas_concs_gpu;
};

class Gas_concs_gpu
{
  public:
    Gas_concs_gpu() = default;
    explicit Gas_concs_gpu(const Gas_concs& ref)
    {
        for (const auto& kv : ref.gas_concs_map) gas_concs_map.emplace(kv.first, Array_gpu<Float, 2>(kv.second));
    }

    const Array_gpu<Float, 2>& get_vmr(const std::string& name) const
    {
        auto it = gas_concs_map.find(name);
        if (it == gas_concs_map.end()) throw std::runtime_error("Gas " + name + " is not available");
        return it->second;
    }
    void set_vmr(const std::string& name, const Array<Float, 2>& data)
    {
        gas_concs_map.erase(name);
        gas_concs_map.emplace(name, Array_gpu<Float, 2>(data));
    }
    void set_vmr(const std::string& name, const Array_gpu<Float, 2>& data)
    {
        gas_concs_map.erase(name);
        gas_concs_map.emplace(name, Array_gpu<Float, 2>(data));
    }
    Bool exists(const std::string& name) const { return gas_concs_map.count(name) != 0; }

    // Names of all gases present (the "available gases" of a k-distribution constructor).
    std::vector<std::string> get_gas_names() const
    {
        std::vector<std::string> n;
        for (const auto& kv : gas_concs_map) n.push_back(kv.first);
        return n;
    }

    // C-ABI descriptors of every gas; the pointers stay valid while this object lives.
    std::vector<rrtmgp_b200_gas_conc> descriptors() const
    {
        std::vector<rrtmgp_b200_gas_conc> d;
        for (const auto& kv : gas_concs_map) {
            rrtmgp_b200_gas_conc c;
            c.name = kv.first.c_str();
            c.vmr = kv.second.ptr();
            c.dim1 = kv.second.dim(1);
            c.dim2 = kv.second.dim(2);
            d.push_back(c);
        }
        return d;
    }

  private:
    std::map<std::string, Array_gpu<Float, 2>> gas_concs_map;
};

#endif
