// Test-infrastructure only: a Python module that compiles DUCC's own NUFFT,
// w-gridder and spherical-harmonic bindings (python/nufft_pymod.cc,
// python/wgridder_pymod.cc, python/sht_pymod.cc) from the reference sources
// where they lie,
// plus a few read-only probes that expose DUCC's internal index computation
// (getpix, tile keys, the stable bucket-sort permutation), its kernel choice,
// its piecewise-polynomial kernel coefficients and its correction factors.
//
// Nothing in the product links or imports this module.  The probes pin the
// CPU restatement in oracle/ and the CUDA path bit-exactly against:
//   - Nufft_ancestor::getpix            src/ducc0/nufft/nufft.h:285-298
//   - get_tile / build_index (1D/2D/3D)  src/ducc0/nufft/nufft.h:301-320,
//                                        :892-907, :1364-1381, :1862-1892
//   - bucket_sort2                      src/ducc0/infra/bucket_sort.h:170
//   - findNufftParameters               src/ducc0/nufft/nufft.h:155-208
//                                        (also alone: params_probe)
//   - selectKernel / getCoeffs          src/ducc0/math/gridding_kernel.cc:28-76,1552
//   - Nufft_ancestor ctor corfac        src/ducc0/nufft/nufft.h:426-431
//
// Build recipe: oracle/Makefile (reads the reference tree, writes oracle/_ref/).

#include <cstdint>
#include <vector>
#include <array>
#include <string>

#include "ducc0/infra/string_utils.cc"
#include "ducc0/infra/threading.cc"
#include "ducc0/infra/mav.cc"
#include "ducc0/math/gl_integrator.cc"
#include "ducc0/math/gridding_kernel.cc"
#include "ducc0/wgridder/wgridder.cc"
#include "ducc0/sht/sht.cc"
#include "ducc0/healpix/healpix_tables.cc"
#include "ducc0/healpix/healpix_base.cc"
#include "ducc0/math/geom_utils.cc"
#include "ducc0/math/space_filling.cc"
#include "ducc0/math/pointing.cc"

#include <pybind11/pybind11.h>
#include <pybind11/numpy.h>
#include <pybind11/stl.h>
#include "ducc0/fft/fft1d_impl.h"
#include "ducc0/fft/fftnd_impl.h"
#include "python/nufft_pymod.cc"
#include "python/wgridder_pymod.cc"
#include "python/sht_pymod.cc"

namespace py = pybind11;
using namespace ducc0;

namespace probe {

template<typename Tcalc, typename Tcoord, size_t ndim>
struct IndexProbe : public detail_nufft::Nufft<Tcalc, Tcalc, Tcoord, ndim>
  {
  using Base = detail_nufft::Nufft<Tcalc, Tcalc, Tcoord, ndim>;
  using Anc = detail_nufft::Nufft_ancestor<Tcalc, Tcalc, ndim>;
  using Base::Base;

  py::dict collect(const cmav<Tcoord,2> &coords)
    {
    size_t npts = coords.shape(0);
    py::dict res;
    std::vector<size_t> nover(ndim);
    for (size_t i=0; i<ndim; ++i) nover[i] = this->Anc::nover[i];
    res["nover"] = nover;
    res["supp"] = this->Anc::supp;
    res["nsafe"] = this->Anc::nsafe;
    res["log2tile"] = int(Anc::log2tile);
    std::vector<double> shift(ndim);
    std::vector<int> maxi0(ndim);
    for (size_t i=0; i<ndim; ++i)
      { shift[i] = this->Anc::shift[i]; maxi0[i] = this->Anc::maxi0[i]; }
    res["shift"] = shift;
    res["maxi0"] = maxi0;
    // permutation produced by build_index + bucket_sort2
    py::array_t<uint32_t> idx(npts);
    auto pidx = idx.mutable_data();
    for (size_t i=0; i<npts; ++i) pidx[i] = this->Anc::coord_idx[i];
    res["coord_idx"] = idx;
    // getpix results per point, in input order
    py::array_t<int32_t> i0arr({npts, ndim});
    py::array_t<double> fracarr({npts, ndim});
    auto pi0 = i0arr.mutable_data();
    auto pfr = fracarr.mutable_data();
    for (size_t i=0; i<npts; ++i)
      {
      std::array<double,ndim> in, frac;
      std::array<int,ndim> i0;
      for (size_t d=0; d<ndim; ++d) in[d] = coords(i,d);
      this->Anc::template getpix<Tcoord>(in, frac, i0);
      for (size_t d=0; d<ndim; ++d)
        { pi0[i*ndim+d] = i0[d]; pfr[i*ndim+d] = frac[d]; }
      }
    res["i0"] = i0arr;
    res["frac"] = fracarr;
    // kernel polynomial and correction factors
    auto krn = this->Anc::krn;
    res["coeff"] = krn->Coeff();
    res["degree"] = krn->degree();
    std::vector<std::vector<double>> cf;
    for (const auto &v: this->Anc::corfac) cf.push_back(v);
    res["corfac"] = cf;
    return res;
    }
  };

template<typename Tcalc, typename Tcoord, size_t ndim>
py::dict run_probe(const py::array &coord_, const std::vector<size_t> &shape,
  double epsilon, bool gridding, size_t nthreads, double sigma_min,
  double sigma_max, const std::vector<double> &periodicity, bool fft_order)
  {
  auto coord = to_cmav<Tcoord,2>(coord_);
  std::array<size_t,ndim> shp;
  for (size_t i=0; i<ndim; ++i) shp[i] = shape[i];
  IndexProbe<Tcalc,Tcoord,ndim> p(gridding, coord, shp, epsilon, nthreads,
    sigma_min, sigma_max, periodicity, fft_order);
  auto res = p.collect(coord);
  // which KernelDB row was chosen
  std::vector<size_t> tdims(shape.begin(), shape.end());
  auto [kidx, dims] = detail_nufft::findNufftParameters<Tcalc,Tcalc>
    (epsilon, sigma_min, sigma_max, tdims, coord.shape(0), gridding,
     adjust_nthreads(nthreads));
  const auto &kp = getKernel(kidx);
  res["kernel_index"] = kidx;
  res["W"] = kp.W;
  res["ofactor"] = kp.ofactor;
  res["kernel_epsilon"] = kp.epsilon;
  res["beta"] = kp.beta;
  res["e0"] = kp.e0;
  return res;
  }

py::dict index_probe(const py::array &coord, const std::vector<size_t> &shape,
  double epsilon, bool singleprec, bool gridding, size_t nthreads,
  double sigma_min, double sigma_max, const std::vector<double> &periodicity,
  bool fft_order)
  {
  size_t ndim = shape.size();
  bool c32 = py::isinstance<py::array_t<float>>(coord);
#define DISPATCH(TC, TK, ND) \
  return run_probe<TC, TK, ND>(coord, shape, epsilon, gridding, nthreads, \
    sigma_min, sigma_max, periodicity, fft_order);
  if (singleprec)
    {
    if (c32)
      { if (ndim==1) DISPATCH(float,float,1) if (ndim==2) DISPATCH(float,float,2) if (ndim==3) DISPATCH(float,float,3) }
    else
      { if (ndim==1) DISPATCH(float,double,1) if (ndim==2) DISPATCH(float,double,2) if (ndim==3) DISPATCH(float,double,3) }
    }
  else
    {
    if (c32)
      { if (ndim==1) DISPATCH(double,float,1) if (ndim==2) DISPATCH(double,float,2) if (ndim==3) DISPATCH(double,float,3) }
    else
      { if (ndim==1) DISPATCH(double,double,1) if (ndim==2) DISPATCH(double,double,2) if (ndim==3) DISPATCH(double,double,3) }
    }
#undef DISPATCH
  MR_fail("unsupported probe combination");
  }

// DUCC's parameter choice alone (findNufftParameters, nufft.h:155-216) for a
// transform of npoints points: kernel row, support, oversampling factor and
// oversampled sizes, without building a plan.
py::dict params_probe(const std::vector<size_t> &shape, size_t npoints, double epsilon,
  bool singleprec, bool gridding, size_t nthreads, double sigma_min, double sigma_max)
  {
  auto [kidx, dims] = singleprec ?
    detail_nufft::findNufftParameters<float,float>(epsilon, sigma_min, sigma_max,
      shape, npoints, gridding, adjust_nthreads(nthreads)) :
    detail_nufft::findNufftParameters<double,double>(epsilon, sigma_min, sigma_max,
      shape, npoints, gridding, adjust_nthreads(nthreads));
  const auto &kp = getKernel(kidx);
  py::dict res;
  res["kernel_index"] = kidx;
  res["W"] = kp.W;
  res["ofactor"] = kp.ofactor;
  res["nover"] = std::vector<size_t>(dims.begin(), dims.end());
  res["nthreads_used"] = adjust_nthreads(nthreads);
  return res;
  }

// Kernel DB rows, for pinning the product's embedded parameter table.
py::list kernel_db()
  {
  py::list out;
  for (const auto &k: detail_gridding_kernel::KernelDB)
    out.append(py::make_tuple(k.W, k.ofactor, k.epsilon, k.beta, k.e0,
                              k.ndim, k.singleprec));
  return out;
  }

// Polynomial coefficients + GL correction data for one DB row.
py::dict kernel_row(size_t idx)
  {
  auto krn = selectKernel(idx);
  py::dict res;
  res["coeff"] = krn->Coeff();
  res["degree"] = krn->degree();
  res["W"] = krn->support();
  res["x"] = krn->Corr().X();
  res["wgtpsi"] = krn->Corr().Wgtpsi();
  return res;
  }

py::dict good_size(size_t n)
  {
  py::dict res;
  res["good_size_complex"] = detail_fft::util1d::good_size_cmplx(n);
  return res;
  }

} // namespace probe

PYBIND11_MODULE(MODNAME, m)
  {
  using namespace pybind11::literals;
  add_nufft(m);
  add_wgridder(m);
  add_sht(m);
  m.def("index_probe", &probe::index_probe, py::kw_only(), "coord"_a,
        "shape"_a, "epsilon"_a, "singleprec"_a, "gridding"_a, "nthreads"_a=1,
        "sigma_min"_a=1.2, "sigma_max"_a=2.51, "periodicity"_a,
        "fft_order"_a=false);
  m.def("params_probe", &probe::params_probe, py::kw_only(), "shape"_a, "npoints"_a,
        "epsilon"_a, "singleprec"_a, "gridding"_a, "nthreads"_a=1, "sigma_min"_a=1.2,
        "sigma_max"_a=2.51);
  m.def("kernel_db", &probe::kernel_db);
  m.def("kernel_row", &probe::kernel_row);
  m.def("good_size", &probe::good_size);
  }
