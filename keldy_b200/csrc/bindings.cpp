// Python bindings of the C++ host classes (include/keldy_b200.hpp) under keldy's Python
// names (python/keldy/common_desc.py, warpers_desc.py, impurity_oneband_desc.py).
#include <pybind11/complex.h>
#include <pybind11/functional.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "keldy_b200.hpp"

namespace py = pybind11;
using namespace keldy;
using namespace keldy::warpers;
using namespace keldy::impurity_oneband;

namespace {

template <typename W, typename C> void warper_methods(C &c) {
  c.def("map_reverse", &W::map_reverse, py::arg("li_vec"))
      .def("map_forward", &W::map_forward, py::arg("ui_vec"))
      .def("ui_from_li", &W::ui_from_li, py::arg("li_vec"))
      .def("li_from_ui", &W::li_from_ui, py::arg("ui_vec"))
      .def("jacobian_reverse", &W::jacobian_reverse, py::arg("li_vec"))
      .def("jacobian_forward", &W::jacobian_forward, py::arg("ui_vec"));
}

std::vector<dcomplex> to_cvec(py::array_t<std::complex<double>, py::array::c_style | py::array::forcecast> a) {
  return std::vector<dcomplex>(a.data(), a.data() + a.size());
}

template <typename T, typename C> void integrator_methods(C &c) {
  c.def_readwrite("warper", &T::warper)
      .def("evaluate_warped_integrand",
           py::overload_cast<std::vector<double> const &, int, bool>(&T::evaluate_warped_integrand, py::const_),
           py::arg("li_vec"), py::arg("start_domain_nr"), py::arg("keep_u_hypercube") = true)
      .def("evaluate_warped_integrand",
           py::overload_cast<std::vector<double> const &>(&T::evaluate_warped_integrand, py::const_),
           py::arg("li_vec"))
      .def("run", &T::run, py::arg("nr_steps"), py::call_guard<py::gil_scoped_release>())
      .def("reset_rng", &T::reset_rng, py::arg("rng_name"), py::arg("rng_state_seed"), py::arg("do_shift") = false,
           py::arg("do_scramble") = false, py::arg("rng_seed_shift") = 0)
      .def("reduce_result", &T::reduce_result)
      .def("reduce_nr_points_run", &T::reduce_nr_points_run)
      .def("reduce_nr_points_in_domain", &T::reduce_nr_points_in_domain)
      .def("get_integrand", &T::get_integrand)
      .def("get_warper", &T::get_warper);
}

} // namespace

PYBIND11_MODULE(_keldy, m) {
  m.doc() = "keldy's Python interface for its QMC hot path, on keldy_b200's sm_100a kernels";

  // ------------------------------------------------------------- common
  py::enum_<spin_t>(m, "spin_t").value("up", up).value("down", down).export_values();
  py::enum_<keldysh_idx_t>(m, "keldysh_idx_t").value("forward", forward).value("backward", backward).export_values();

  py::class_<contour_pt_t>(m, "ContourPtT", "Point of the Keldysh Contour (time, keldysh_idx, timesplit)")
      .def(py::init<>())
      .def(py::init([](double t, int k, int s) { return contour_pt_t{t, keldysh_idx_t(k), s}; }), py::arg("time"),
           py::arg("k_idx"), py::arg("timesplit_n") = 0)
      .def_readwrite("time", &contour_pt_t::time)
      .def_property(
          "k_idx", [](contour_pt_t const &c) { return int(c.k_idx); },
          [](contour_pt_t &c, int k) { c.k_idx = keldysh_idx_t(k); })
      .def_readwrite("timesplit_n", &contour_pt_t::timesplit_n)
      .def("__eq__", &contour_pt_t::operator==);
  m.def("compare_3way", &compare_3way, py::arg("a"), py::arg("b"));

  py::class_<sobol>(m, "Sobol")
      .def(py::init<int, int, int>(), py::arg("dim"), py::arg("rng_state_seed"), py::arg("log_max_points_") = 31)
      .def(py::init<int, int, bool, bool, int, int>(), py::arg("dim"), py::arg("rng_state_seed"), py::arg("do_shift"),
           py::arg("do_scramble"), py::arg("rng_seed_shift"), py::arg("log_max_points_") = 31)
      .def("__call__", &sobol::operator())
      .def("seed", &sobol::seed, py::arg("k"))
      .def("discard", &sobol::discard, py::arg("nr_discard"))
      .def(
          "points",
          [](sobol &s, int64_t count) {
            std::vector<double> v = s.points(count);
            py::array_t<double> a({(py::ssize_t)count, (py::ssize_t)s.dimension()});
            std::copy(v.begin(), v.end(), a.mutable_data());
            return a;
          },
          py::arg("count"), "the next `count` points as a [count, dim] array (one device launch)");

  // ------------------------------------------------------------ warpers
  auto wi = py::class_<warper_identity_t>(m, "WarperIdentityT").def(py::init<>());
  warper_methods<warper_identity_t>(wi);
  auto wp = py::class_<warper_plasma_uv_t>(m, "WarperPlasmaUvT").def(py::init<double>(), py::arg("t_max_"));
  warper_methods<warper_plasma_uv_t>(wp);
  auto ws = py::class_<warper_product_1d_simple_t>(m, "WarperProduct1dSimpleT")
                .def(py::init<>())
                .def(py::init([](py::object, py::object, py::object, double, bool) -> warper_product_1d_simple_t {
                       throw std::runtime_error(
                           "WarperProduct1dSimpleT from Python functions has no device form; use "
                           "make_product_1d_simple_exponential/inverse/inverse_square/inverse_power/uniform");
                     }),
                     py::arg("f1_"), py::arg("f1_integrated_"), py::arg("f1_integrated_inverse_"),
                     py::arg("domain_u_max_"), py::arg("do_domain_checks") = true)
                .def("__call__", &warper_product_1d_simple_t::operator(), py::arg("ui_vec"));
  warper_methods<warper_product_1d_simple_t>(ws);
  m.def("make_product_1d_simple_exponential", &make_product_1d_simple_exponential, py::arg("domain_u_max"),
        py::arg("w_scale"));
  m.def("make_product_1d_simple_inverse", &make_product_1d_simple_inverse, py::arg("domain_u_max"), py::arg("w_scale"));
  m.def("make_product_1d_simple_inverse_square", &make_product_1d_simple_inverse_square, py::arg("domain_u_max"),
        py::arg("w_scale"));
  m.def("make_product_1d_simple_inverse_power", &make_product_1d_simple_inverse_power, py::arg("power"),
        py::arg("domain_u_max"), py::arg("w_scale"));
  m.def("make_product_1d_simple_uniform", &make_product_1d_simple_uniform, py::arg("domain_u_max"));
  auto wtn = py::class_<warper_product_1d_simple_interp_nearest_t>(m, "WarperProduct1dSimpleInterpNearestT")
                 .def(py::init<std::vector<double>, std::vector<double>>(), py::arg("times_u_pts"), py::arg("f1_pts"))
                 .def(py::init<std::function<double(double)> const &, double, int>(), py::arg("f1_"),
                      py::arg("domain_u_max_"), py::arg("nr_sample_points_"))
                 .def("get_times_u_pts", &warper_product_1d_simple_interp_nearest_t::get_times_u_pts)
                 .def("get_f1_pts", &warper_product_1d_simple_interp_nearest_t::get_f1_pts);
  warper_methods<warper_product_1d_simple_interp_nearest_t>(wtn);
  auto wpn = py::class_<warper_product_1d_interp_nearest_t>(m, "WarperProduct1dInterpNearestT")
                 .def(py::init<>())
                 .def("reserve", &warper_product_1d_interp_nearest_t::reserve, py::arg("new_cap"))
                 .def("size", &warper_product_1d_interp_nearest_t::size)
                 .def("emplace_back", &warper_product_1d_interp_nearest_t::emplace_back, py::arg("w"))
                 .def("get_1d_warper", &warper_product_1d_interp_nearest_t::get_1d_warper, py::arg("axis"));
  warper_methods<warper_product_1d_interp_nearest_t>(wpn);
  auto wpa = py::class_<warper_product_1d_t>(m, "WarperProduct1dT")
                 .def(py::init<>())
                 .def("reserve", &warper_product_1d_t::reserve, py::arg("new_cap"))
                 .def("size", &warper_product_1d_t::size)
                 .def("emplace_back", &warper_product_1d_t::emplace_back, py::arg("w"))
                 .def("get_1d_warper", &warper_product_1d_t::get_1d_warper, py::arg("axis"));
  warper_methods<warper_product_1d_t>(wpa);
  m.def("make_product_1d_inverse_cube_alternate", &make_product_1d_inverse_cube_alternate, py::arg("order"),
        py::arg("time"), py::arg("warper_scale"));
  m.def("make_product_1d_inverse_cube_alternate_interp_nearest", &make_product_1d_inverse_cube_alternate_interp_nearest,
        py::arg("order"), py::arg("time"), py::arg("warper_scale"), py::arg("nr_sample_points_warper"));
  // f1_: the closed form of f1 by name (the device has no Python); w_scale, power its parameters
  auto wth =
      py::class_<warper_product_1d_simple_interp_hybrid_t>(m, "WarperProduct1dSimpleInterpHybridT")
          .def(py::init([](py::object f1, double domain_u_max, int n, double w_scale, int power) {
                 if (!py::isinstance<py::str>(f1))
                   throw std::runtime_error("WarperProduct1dSimpleInterpHybridT needs f1 in closed form on the GPU: "
                                            "'exponential', 'inverse', 'inverse_square', 'inverse_power' or "
                                            "'uniform' (with w_scale, power)");
                 const std::string name = f1.cast<std::string>();
                 int kind = name == "exponential"      ? KB_WARPER_EXPONENTIAL
                            : name == "inverse"        ? KB_WARPER_INVERSE
                            : name == "inverse_square" ? KB_WARPER_INVERSE_SQUARE
                            : name == "inverse_power"  ? KB_WARPER_INVERSE_POWER
                            : name == "uniform"        ? KB_WARPER_UNIFORM
                                                       : -1;
                 if (kind < 0) throw std::runtime_error("unknown f1 closed form '" + name + "'");
                 return warper_product_1d_simple_interp_hybrid_t(kb_warper{kind, power, domain_u_max, w_scale}, n);
               }),
               py::arg("f1_"), py::arg("domain_u_max_"), py::arg("nr_sample_points_"), py::arg("w_scale") = 1.0,
               py::arg("power") = 1);
  warper_methods<warper_product_1d_simple_interp_hybrid_t>(wth);
  auto wph = py::class_<warper_product_1d_interp_hybrid_t>(m, "WarperProduct1dInterpHybridT")
                 .def(py::init<>())
                 .def("reserve", &warper_product_1d_interp_hybrid_t::reserve, py::arg("new_cap"))
                 .def("size", &warper_product_1d_interp_hybrid_t::size)
                 .def("emplace_back", &warper_product_1d_interp_hybrid_t::emplace_back, py::arg("w"))
                 .def("get_1d_warper", &warper_product_1d_interp_hybrid_t::get_1d_warper, py::arg("axis"));
  warper_methods<warper_product_1d_interp_hybrid_t>(wph);
  m.def("make_product_1d_inverse_cube_alternate_interp_hybrid", &make_product_1d_inverse_cube_alternate_interp_hybrid,
        py::arg("order"), py::arg("time"), py::arg("warper_scale"), py::arg("nr_sample_points_warper"));
  py::class_<projection_bins>(m, "ProjectionBins")
      .def("get_data", &projection_bins::get_data)
      .def("get_nr_values_added", &projection_bins::get_nr_values_added)
      .def("get_nr_bins", &projection_bins::get_nr_bins)
      .def("get_bin_size", &projection_bins::get_bin_size)
      .def("get_bin_coord", &projection_bins::get_bin_coord);
  auto wpr = py::class_<warper_projection_t>(m, "WarperProjectionT")
                 .def(py::init<std::function<dcomplex(std::vector<double>)> const &, int, int, int, double, bool>(),
                      py::arg("warped_integrand"), py::arg("order"), py::arg("num_bins"), py::arg("nr_samples"),
                      py::arg("sigma"), py::arg("optimize_sigma") = true)
                 .def("get_xi", &warper_projection_t::get_xi, py::arg("axis"))
                 .def("get_sigmas", &warper_projection_t::get_sigmas)
                 .def("get_fi", &warper_projection_t::get_fi, py::arg("axis"));
  warper_methods<warper_projection_t>(wpr);
  m.def("vi_from_ui", &vi_from_ui, py::arg("t_max"), py::arg("u_times"));
  m.def("ui_from_vi", &ui_from_vi, py::arg("t_max"), py::arg("v_times"));

  py::class_<warper_train_t>(m, "WarperTrainT")
      .def(py::init<>())
      .def("emplace_back", [](warper_train_t &t, warper_identity_t const &w) { t.emplace_back(w); }, py::arg("w"))
      .def("emplace_back", [](warper_train_t &t, warper_plasma_uv_t const &w) { t.emplace_back(w); }, py::arg("w"))
      .def("emplace_back", [](warper_train_t &t, warper_product_1d_simple_t const &w) { t.emplace_back(w); },
           py::arg("w"))
      .def("emplace_back",
           [](warper_train_t &t, warper_product_1d_simple_interp_nearest_t const &w) { t.emplace_back(w); },
           py::arg("w"))
      .def("emplace_back", [](warper_train_t &t, warper_product_1d_interp_nearest_t const &w) { t.emplace_back(w); },
           py::arg("w"))
      .def("emplace_back", [](warper_train_t &t, warper_product_1d_t const &w) { t.emplace_back(w); }, py::arg("w"))
      .def("emplace_back",
           [](warper_train_t &t, warper_product_1d_simple_interp_hybrid_t const &w) { t.emplace_back(w); },
           py::arg("w"))
      .def("emplace_back", [](warper_train_t &t, warper_product_1d_interp_hybrid_t const &w) { t.emplace_back(w); },
           py::arg("w"))
      .def("emplace_back", [](warper_train_t &t, warper_projection_t const &w) { t.emplace_back(w); }, py::arg("w"))
      .def("reserve", &warper_train_t::reserve, py::arg("new_cap"))
      .def("clear", &warper_train_t::clear)
      .def("size", &warper_train_t::size)
      .def("__len__", &warper_train_t::size)
      .def("map_reverse",
           py::overload_cast<std::vector<double> const &, int, int>(&warper_train_t::map_reverse, py::const_),
           py::arg("li_vec"), py::arg("start_domain_nr"), py::arg("end_domain_nr"))
      .def("map_reverse", py::overload_cast<std::vector<double> const &>(&warper_train_t::map_reverse, py::const_),
           py::arg("li_vec"))
      .def("map_forward",
           py::overload_cast<std::vector<double> const &, int, int>(&warper_train_t::map_forward, py::const_),
           py::arg("ui_vec"), py::arg("start_domain_nr"), py::arg("end_domain_nr"))
      .def("map_forward", py::overload_cast<std::vector<double> const &>(&warper_train_t::map_forward, py::const_),
           py::arg("ui_vec"))
      .def("ui_from_li", &warper_train_t::ui_from_li, py::arg("li_vec"))
      .def("li_from_ui", &warper_train_t::li_from_ui, py::arg("ui_vec"))
      .def("jacobian_reverse", &warper_train_t::jacobian_reverse, py::arg("li_vec"))
      .def("jacobian_forward", &warper_train_t::jacobian_forward, py::arg("ui_vec"));

  // ------------------------------------------------- impurity_oneband
  py::class_<gf_index_t>(m, "GfIndexT")
      .def(py::init<>())
      .def(py::init<double, int, int>(), py::arg("time_"), py::arg("spin_"), py::arg("k_idx_"))
      .def(py::init<double, int, int, int>(), py::arg("time_"), py::arg("spin_"), py::arg("k_idx_"),
           py::arg("timesplit_n_"))
      .def(py::init<double, int, int, int, int>(), py::arg("time_"), py::arg("spin_"), py::arg("k_idx_"),
           py::arg("timesplit_n_"), py::arg("orbital_"))
      .def_readwrite("contour", &gf_index_t::contour)
      .def_property(
          "spin", [](gf_index_t const &g) { return int(g.spin); }, [](gf_index_t &g, int s) { g.spin = spin_t(s); })
      .def_readwrite("orbital", &gf_index_t::orbital);

  m.attr("FT_SYMMETRIC") = KB_FT_SYMMETRIC;
  m.attr("FT_MIRROR") = KB_FT_MIRROR;
  py::class_<g0_model>(m, "G0ModelTables", py::dynamic_attr(),
                       "g0 tables on the device (spin up, orbital (0,0) plus optional blocks)")
      .def_static(
          "from_tables",
          [](double time_max, py::array_t<std::complex<double>> lesser, py::array_t<std::complex<double>> greater,
             double alpha) { return g0_model::from_tables(time_max, to_cvec(lesser), to_cvec(greater), alpha); },
          py::arg("time_max"), py::arg("lesser"), py::arg("greater"), py::arg("alpha") = 0.0)
      .def(
          "set_table",
          [](g0_model &g, int spin, int o1, int o2, py::array_t<std::complex<double>> lesser,
             py::array_t<std::complex<double>> greater) { g.set_table(spin, o1, o2, to_cvec(lesser), to_cvec(greater)); },
          py::arg("spin"), py::arg("o1"), py::arg("o2"), py::arg("lesser"), py::arg("greater"))
      .def_static("empty", &g0_model::empty, py::arg("time_max"), py::arg("npts"), py::arg("alpha") = 0.0)
      .def("set_interpolation", &g0_model::set_interpolation, py::arg("order"))
      .def(
          "set_fourier",
          [](g0_model &g, int o1, int o2, py::array_t<double> w, py::array_t<std::complex<double>> cl,
             py::array_t<std::complex<double>> cg, int flags) {
            auto wr = w.unchecked<1>();
            std::vector<double> wv((size_t)wr.shape(0));
            for (py::ssize_t k = 0; k < wr.shape(0); ++k) wv[(size_t)k] = wr(k);
            g.set_fourier(o1, o2, wv, to_cvec(cl), to_cvec(cg), flags);
          },
          py::arg("o1"), py::arg("o2"), py::arg("w"), py::arg("cl"), py::arg("cg"), py::arg("flags"))
      .def(
          "set_fft",
          [](g0_model &g, int o1, int o2, py::array_t<std::complex<double>> gl, py::array_t<std::complex<double>> gg,
             int flags) { g.set_fft(o1, o2, to_cvec(gl), to_cvec(gg), flags); },
          py::arg("o1"), py::arg("o2"), py::arg("gl"), py::arg("gg"), py::arg("flags") = 0)
      .def(
          "set_rational",
          [](g0_model &g, int o1, int o2, py::list terms, double beta, int flags) {
            std::vector<double> mu;
            std::vector<std::vector<dcomplex>> z, r;
            for (auto item : terms) {
              auto t = item.cast<py::tuple>();
              mu.push_back(t[0].cast<double>());
              z.push_back(to_cvec(t[1].cast<py::array_t<std::complex<double>>>()));
              r.push_back(to_cvec(t[2].cast<py::array_t<std::complex<double>>>()));
            }
            g.set_rational(o1, o2, mu, z, r, beta, flags);
          },
          py::arg("o1"), py::arg("o2"), py::arg("terms"), py::arg("beta"), py::arg("flags") = 0)
      .def(
          "get_table",
          [](g0_model const &g, int spin, int o1, int o2) {
            auto t = g.get_table(spin, o1, o2);
            py::array_t<std::complex<double>> l((py::ssize_t)t.first.size()), r((py::ssize_t)t.second.size());
            std::copy(t.first.begin(), t.first.end(), l.mutable_data());
            std::copy(t.second.begin(), t.second.end(), r.mutable_data());
            return py::make_tuple(l, r);
          },
          py::arg("spin"), py::arg("o1"), py::arg("o2"))
      .def_readwrite("make_dot_lead", &g0_model::make_dot_lead)
      .def_property_readonly("time_max", &g0_model::time_max)
      .def_property_readonly("npts", &g0_model::npts)
      .def_property_readonly("alpha", &g0_model::alpha);

  py::class_<g0_keldysh_contour_t>(m, "G0KeldyshContourT")
      .def(py::init<g0_model>(), py::arg("model_"))
      .def_readwrite("model", &g0_keldysh_contour_t::model)
      .def("__call__", &g0_keldysh_contour_t::operator(), py::arg("a"), py::arg("b"), py::arg("internal_point") = true)
      .def("get_time_max", &g0_keldysh_contour_t::get_time_max);

  py::class_<integrand_g_direct>(m, "IntegrandGDirect")
      .def(py::init<g0_keldysh_contour_t, gf_index_t, gf_index_t, double>(), py::arg("g0_"), py::arg("external_A_"),
           py::arg("external_B_"), py::arg("cutoff_") = 0.)
      .def("__call__", &integrand_g_direct::operator(), py::arg("times"), py::arg("keep_u_hypercube") = true)
      .def("eval_no_det", &integrand_g_direct::eval_no_det, py::arg("times"), py::arg("keep_u_hypercube") = true)
      .def("set_algorithm", &integrand_g_direct::set_algorithm, py::arg("algo"))
      .def(
          "evaluate_batch",
          [](integrand_g_direct const &f, py::array_t<double, py::array::c_style | py::array::forcecast> times,
             bool keep) {
            if (times.ndim() != 2) throw std::runtime_error("times must be a [count, order] array");
            const int64_t count = times.shape(0);
            std::vector<dcomplex> vals;
            std::vector<int> dom;
            f.eval_many((int)times.shape(1), count, times.data(), vals, dom, keep);
            py::array_t<std::complex<double>> out(count);
            py::array_t<int> pdom(count);
            std::copy(vals.begin(), vals.end(), out.mutable_data());
            std::copy(dom.begin(), dom.end(), pdom.mutable_data());
            return py::make_tuple(out, pdom);
          },
          py::arg("times"), py::arg("keep_u_hypercube") = true,
          "the integrand at many time vectors in one device launch: (values, in_domain)");

  auto cq = py::class_<compute_charge_Q_direct>(m, "ComputeChargeQDirect")
                .def(py::init<g0_model, double, int, double>(), py::arg("model"), py::arg("time"), py::arg("order"),
                     py::arg("cutoff_integrand"));
  integrator_methods<compute_charge_Q_direct>(cq);
  auto cj = py::class_<compute_current_J_direct>(m, "ComputeCurrentJDirect")
                .def(py::init<g0_model, double, int, double>(), py::arg("model"), py::arg("time"), py::arg("order"),
                     py::arg("cutoff_integrand"));
  integrator_methods<compute_current_J_direct>(cj);
  py::class_<binner_1d>(m, "BinnerT1")
      .def(py::init<double, double, long>(), py::arg("xmin"), py::arg("xmax"), py::arg("nr_bins"))
      .def("get_data", &binner_1d::get_data)
      .def("get_nr_values_added", &binner_1d::get_nr_values_added)
      .def("get_nr_values_dropped", &binner_1d::get_nr_values_dropped)
      .def("get_nr_bins", &binner_1d::get_nr_bins)
      .def("get_bin_size", &binner_1d::get_bin_size)
      .def("get_bin_coord", &binner_1d::get_bin_coord);
  auto cqt = py::class_<compute_charge_Q_direct_time>(m, "ComputeChargeQDirectTime")
                 .def(py::init<g0_model, double, int, int, double>(), py::arg("model"), py::arg("time"),
                      py::arg("order"), py::arg("nr_time_slices"), py::arg("cutoff_integrand"));
  integrator_methods<compute_charge_Q_direct_time>(cqt);
  m.def(
      "make_warper_from_proj",
      [](compute_charge_Q_direct const &c, int order, int num_bins, int nr_samples, double sigma, bool keep) {
        return keldy::warpers::make_warper_from_proj(c, order, num_bins, nr_samples, sigma, keep);
      },
      py::arg("computer"), py::arg("order"), py::arg("num_bins"), py::arg("nr_samples"), py::arg("sigma"),
      py::arg("keep_u_hypercube") = true);
  m.def(
      "make_warper_from_proj",
      [](std::function<dcomplex(std::vector<double>)> const &f, int order, int num_bins, int nr_samples,
         double sigma) { return keldy::warpers::make_warper_from_proj(f, order, num_bins, nr_samples, sigma); },
      py::arg("warped_integrand"), py::arg("order"), py::arg("num_bins"), py::arg("nr_samples"), py::arg("sigma"));
  m.def(
      "make_projection_warper",
      [](compute_charge_Q_direct const &c, int order, int num_bins, int nr_samples, double sigma, bool optimize,
         bool keep) {
        return keldy::warpers::make_projection_warper(c, order, num_bins, nr_samples, sigma, optimize, keep);
      },
      py::arg("computer"), py::arg("order"), py::arg("num_bins"), py::arg("nr_samples"), py::arg("sigma"),
      py::arg("optimize_sigma") = true, py::arg("keep_u_hypercube") = true);
  py::class_<binner_2d>(m, "BinnerT11")
      .def(py::init<double, double, long>(), py::arg("xmin"), py::arg("xmax"), py::arg("nr_bins"))
      .def("get_data_flat", &binner_2d::get_data_flat)
      .def("get_nr_values_added_flat", &binner_2d::get_nr_values_added_flat)
      .def("get_nr_values_dropped", &binner_2d::get_nr_values_dropped)
      .def("get_nr_bins", &binner_2d::get_nr_bins)
      .def("get_bin_size", &binner_2d::get_bin_size)
      .def("get_bin_coord", &binner_2d::get_bin_coord);
  py::class_<integrand_g_kernel>(m, "IntegrandGKernel")
      .def(py::init<g0_keldysh_contour_t, gf_index_t>(), py::arg("g0"), py::arg("g_idx_X"))
      .def("__call__", &integrand_g_kernel::operator(), py::arg("times"), py::arg("keep_u_hypercube") = true);
  py::class_<compute_gf_kernel>(m, "ComputeGfKernel")
      .def(py::init<g0_model, double, int, int>(), py::arg("model"), py::arg("time"), py::arg("order"),
           py::arg("nr_bins") = 100)
      .def_readwrite("warper", &compute_gf_kernel::warper)
      .def("run", &compute_gf_kernel::run, py::arg("nr_steps"), py::call_guard<py::gil_scoped_release>())
      .def("reset_rng", &compute_gf_kernel::reset_rng, py::arg("rng_name"), py::arg("rng_state_seed"),
           py::arg("do_shift") = false, py::arg("do_scramble") = false, py::arg("rng_seed_shift") = 0)
      .def("reduce_result", &compute_gf_kernel::reduce_result)
      .def("reduce_nr_points_run", &compute_gf_kernel::reduce_nr_points_run)
      .def("reduce_nr_points_in_domain", &compute_gf_kernel::reduce_nr_points_in_domain)
      .def("get_integrand", &compute_gf_kernel::get_integrand)
      .def("get_warper", &compute_gf_kernel::get_warper);
  py::class_<integrand_g_kernel_single_omega>(m, "IntegrandGKernelSingleOmega")
      .def(py::init<g0_keldysh_contour_t, gf_index_t, double>(), py::arg("g0"), py::arg("g_idx_X"), py::arg("omega"))
      .def("__call__", &integrand_g_kernel_single_omega::operator(), py::arg("times"),
           py::arg("keep_u_hypercube") = true);
  py::class_<compute_gf_kernel_single_omega>(m, "ComputeGfKernelSingleOmega")
      .def(py::init<g0_model, double, double, int>(), py::arg("model"), py::arg("time"), py::arg("omega"),
           py::arg("order"))
      .def_readwrite("warper", &compute_gf_kernel_single_omega::warper)
      .def("run", &compute_gf_kernel_single_omega::run, py::arg("nr_steps"), py::call_guard<py::gil_scoped_release>())
      .def("reset_rng", &compute_gf_kernel_single_omega::reset_rng, py::arg("rng_name"), py::arg("rng_state_seed"),
           py::arg("do_shift") = false, py::arg("do_scramble") = false, py::arg("rng_seed_shift") = 0)
      .def("reduce_result", &compute_gf_kernel_single_omega::reduce_result)
      .def("reduce_nr_points_run", &compute_gf_kernel_single_omega::reduce_nr_points_run)
      .def("reduce_nr_points_in_domain", &compute_gf_kernel_single_omega::reduce_nr_points_in_domain)
      .def("get_integrand", &compute_gf_kernel_single_omega::get_integrand)
      .def("get_warper", &compute_gf_kernel_single_omega::get_warper);
}
