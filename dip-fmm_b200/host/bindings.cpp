// pybind11 module `cdfmm`: Python face of cdfmm::UniformFmm on the B200.
//
// Names, argument names, defaults, dtypes and the {"phi", "H"} result dict
// follow upstream python/bindings.cpp (enums :391-413 and :1031-1033,
// UniformFmmOptions :584-599, UniformFmm :601-774, cuda_direct_p2p_reference
// :865-892) so user scripts and the reference's own tests read the same.
// C++ std::invalid_argument surfaces as ValueError, std::runtime_error as
// RuntimeError (pybind11's standard translation, as upstream).
// Additions: ExecutionBackend.CUDA_B200, B200M2L, options.max_states /
// b200_m2l / device, UniformFmm.evaluate_states (K states per call) and
// UniformFmm.evaluate_device (raw device pointers, e.g. torch tensors).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "cdfmm/uniform_fmm.hpp"
#include "cdfmm/uniform_tree.hpp"
#include "cdfmm_b200.h"

namespace py = pybind11;
using namespace cdfmm;

namespace {

using DoubleArray = py::array_t<double, py::array::c_style | py::array::forcecast>;
using FloatArray = py::array_t<float, py::array::c_style | py::array::forcecast>;

std::vector<Vec3> parse_vec3_array(const py::handle &input, const std::string &name) {
  const DoubleArray a = py::cast<DoubleArray>(input);
  if (a.ndim() != 2 || a.shape(1) != 3) throw std::invalid_argument(name + " must have shape (n, 3)");
  const auto v = a.unchecked<2>();
  std::vector<Vec3> out(static_cast<std::size_t>(a.shape(0)));
  for (py::ssize_t i = 0; i < a.shape(0); ++i) out[static_cast<std::size_t>(i)] = {v(i, 0), v(i, 1), v(i, 2)};
  return out;
}

std::vector<Vec3> parse_tree_points(const py::handle &input) {
  if (py::isinstance<py::array>(input)) return parse_vec3_array(input, "points");
  std::vector<Vec3> out;
  for (const auto &item : py::reinterpret_borrow<py::iterable>(input)) {
    if (py::isinstance<Vec3>(item)) {
      out.push_back(py::cast<Vec3>(item));
    } else if (py::isinstance<py::sequence>(item)) {
      const auto s = py::reinterpret_borrow<py::sequence>(item);
      if (s.size() != 3) throw std::invalid_argument("Each point must have exactly three components");
      out.push_back({py::cast<double>(s[0]), py::cast<double>(s[1]), py::cast<double>(s[2])});
    } else {
      throw std::invalid_argument("Points must be Vec3 objects or length-three sequences");
    }
  }
  return out;
}

// A CUDA array (torch tensor, CuPy array, ...) through the CUDA Array
// Interface: its device pointer after checking float32, C-contiguous layout
// and the expected shape (zero-copy device I/O; the reference copies
// element-wise through host memory, python/bindings.cpp:59-80,188-226).
std::uintptr_t cuda_array_ptr(const py::object &a, const std::vector<long> &shape, const char *name) {
  if (!py::hasattr(a, "__cuda_array_interface__"))
    throw std::invalid_argument(std::string(name) + " must be a CUDA array (__cuda_array_interface__)");
  const py::dict cai = a.attr("__cuda_array_interface__");
  const std::string typestr = py::str(cai["typestr"]);
  if (typestr != "<f4") throw std::invalid_argument(std::string(name) + " must be float32");
  const py::tuple sh = cai["shape"];
  if (sh.size() != shape.size()) throw std::invalid_argument(std::string(name) + " has the wrong number of dimensions");
  for (size_t i = 0; i < shape.size(); ++i)
    if (sh[i].cast<long>() != shape[i]) throw std::invalid_argument(std::string(name) + " has the wrong shape");
  if (cai.contains("strides") && !cai["strides"].is_none()) {
    const py::tuple st = cai["strides"];
    long expect = 4;
    for (size_t i = shape.size(); i-- > 0;) {
      if (shape[i] > 1 && st[i].cast<long>() != expect) throw std::invalid_argument(std::string(name) + " must be C-contiguous");
      expect *= shape[i];
    }
  }
  const py::tuple data = cai["data"];
  return data[0].cast<std::uintptr_t>();
}

OutputFlags parse_output(const std::string &output) {
  if (output == "field") return OutputFlags::Field;
  if (output == "potential") return OutputFlags::Potential;
  if (output == "both") return OutputFlags::Both;
  throw std::invalid_argument("output must be 'field', 'potential', or 'both'");
}

std::vector<int> parse_ids(const py::object &ids) {
  if (ids.is_none()) return {};
  return py::cast<std::vector<int>>(ids);
}

py::dict results_to_dict(const std::vector<FloatPotentialField> &r) {
  py::array_t<float> phi(static_cast<py::ssize_t>(r.size()));
  py::array_t<float> H({static_cast<py::ssize_t>(r.size()), static_cast<py::ssize_t>(3)});
  auto p = phi.mutable_unchecked<1>();
  auto h = H.mutable_unchecked<2>();
  for (py::ssize_t i = 0; i < static_cast<py::ssize_t>(r.size()); ++i) {
    const FloatPotentialField &v = r[static_cast<std::size_t>(i)];
    p(i) = v.phi;
    h(i, 0) = v.H.x;
    h(i, 1) = v.H.y;
    h(i, 2) = v.H.z;
  }
  py::dict d;
  d["phi"] = phi;
  d["H"] = H;
  return d;
}

py::array_t<float> floats_to_array(std::span<const float> v) {
  py::array_t<float> a(static_cast<py::ssize_t>(v.size()));
  auto o = a.mutable_unchecked<1>();
  for (py::ssize_t i = 0; i < static_cast<py::ssize_t>(v.size()); ++i) o(i) = v[static_cast<std::size_t>(i)];
  return a;
}

py::array_t<double> points_to_array(std::span<const Vec3> pts) {
  py::array_t<double> a({static_cast<py::ssize_t>(pts.size()), static_cast<py::ssize_t>(3)});
  auto o = a.mutable_unchecked<2>();
  for (py::ssize_t i = 0; i < static_cast<py::ssize_t>(pts.size()); ++i) {
    o(i, 0) = pts[static_cast<std::size_t>(i)].x;
    o(i, 1) = pts[static_cast<std::size_t>(i)].y;
    o(i, 2) = pts[static_cast<std::size_t>(i)].z;
  }
  return a;
}

py::dict phase(const PhaseTiming &t) {
  py::dict d;
  d["total_seconds"] = t.total_seconds;
  d["calls"] = t.calls;
  return d;
}

} // namespace

PYBIND11_MODULE(cdfmm, m) {
  m.doc() = "Cartesian dipole FMM: static-geometry uniform-octree evaluation on NVIDIA B200";

  py::class_<Vec3>(m, "Vec3")
      .def(py::init<double, double, double>())
      .def_readwrite("x", &Vec3::x)
      .def_readwrite("y", &Vec3::y)
      .def_readwrite("z", &Vec3::z);

  py::class_<TreeNode>(m, "TreeNode")
      .def_readonly("index", &TreeNode::index)
      .def_readonly("level", &TreeNode::level)
      .def_readonly("parent", &TreeNode::parent)
      .def_readonly("children", &TreeNode::children)
      .def_readonly("ix", &TreeNode::ix)
      .def_readonly("iy", &TreeNode::iy)
      .def_readonly("iz", &TreeNode::iz)
      .def_readonly("morton_index", &TreeNode::morton_index)
      .def_readonly("centre", &TreeNode::centre)
      .def_readonly("half_width", &TreeNode::half_width)
      .def_readonly("source_begin", &TreeNode::source_begin)
      .def_readonly("source_end", &TreeNode::source_end)
      .def_readonly("target_begin", &TreeNode::target_begin)
      .def_readonly("target_end", &TreeNode::target_end)
      .def_readonly("list1", &TreeNode::list1)
      .def_readonly("list2", &TreeNode::list2)
      .def_property_readonly("source_count", &TreeNode::source_count)
      .def_property_readonly("target_count", &TreeNode::target_count)
      .def_property_readonly("is_leaf", &TreeNode::is_leaf);

  py::class_<UniformTreeOptions>(m, "UniformTreeOptions")
      .def(py::init<>())
      .def_readwrite("max_level", &UniformTreeOptions::max_level)
      .def_readwrite("include_empty_nodes", &UniformTreeOptions::include_empty_nodes)
      .def_readwrite("cubic_root_box", &UniformTreeOptions::cubic_root_box)
      .def_readwrite("root_centre", &UniformTreeOptions::root_centre)
      .def_readwrite("root_half_width", &UniformTreeOptions::root_half_width);

  py::class_<UniformTree>(m, "UniformTree")
      .def(py::init([](py::object s, const UniformTreeOptions &o) { return UniformTree(parse_tree_points(s), o); }),
           py::arg("source_positions"), py::arg("options"))
      .def(py::init([](py::object s, py::object t, const UniformTreeOptions &o) {
             return UniformTree(parse_tree_points(s), parse_tree_points(t), o);
           }),
           py::arg("source_positions"), py::arg("target_positions"), py::arg("options"))
      .def_property_readonly("max_level", &UniformTree::max_level)
      .def_property_readonly("n_levels", &UniformTree::n_levels)
      .def_property_readonly("leaf_level", &UniformTree::leaf_level)
      .def_property_readonly("root_centre", &UniformTree::root_centre)
      .def_property_readonly("root_half_width", &UniformTree::root_half_width)
      .def_property_readonly("nodes", [](const UniformTree &t) {
        return std::vector<TreeNode>(t.nodes().begin(), t.nodes().end());
      })
      .def_property_readonly("source_permutation", [](const UniformTree &t) {
        return std::vector<int>(t.source_permutation().begin(), t.source_permutation().end());
      })
      .def_property_readonly("source_inverse_permutation", [](const UniformTree &t) {
        return std::vector<int>(t.source_inverse_permutation().begin(), t.source_inverse_permutation().end());
      })
      .def_property_readonly("target_permutation", [](const UniformTree &t) {
        return std::vector<int>(t.target_permutation().begin(), t.target_permutation().end());
      })
      .def_property_readonly("target_inverse_permutation", [](const UniformTree &t) {
        return std::vector<int>(t.target_inverse_permutation().begin(), t.target_inverse_permutation().end());
      })
      .def("leaf_indices", [](const UniformTree &t) {
        return std::vector<int>(t.leaf_indices().begin(), t.leaf_indices().end());
      })
      .def("leaf_source_offsets", &UniformTree::leaf_source_offsets,
           "Exclusive prefix of source counts over Morton-ordered leaves (8^max_level + 1 entries).")
      .def("leaf_target_offsets", &UniformTree::leaf_target_offsets)
      .def("leaf_index_for_source", &UniformTree::leaf_index_for_source)
      .def("leaf_index_for_target", &UniformTree::leaf_index_for_target)
      .def("sorted_source_positions", [](const UniformTree &t) { return points_to_array(t.sorted_source_positions()); })
      .def("sorted_target_positions", [](const UniformTree &t) { return points_to_array(t.sorted_target_positions()); });

  py::enum_<M2LBackend>(m, "M2LBackend").value("Static", M2LBackend::Static).value("Reference", M2LBackend::Reference);
  py::enum_<StaticMatrixBackend>(m, "StaticMatrixBackend")
      .value("PORTABLE", StaticMatrixBackend::Portable)
      .value("ONE_MKL", StaticMatrixBackend::OneMkl);
  py::enum_<ExecutionBackend>(m, "ExecutionBackend")
      .value("AUTO", ExecutionBackend::Auto)
      .value("CPU_REFERENCE", ExecutionBackend::CpuReference)
      .value("CPU_STATIC", ExecutionBackend::CpuStatic)
      .value("CUDA_M2L_P2P", ExecutionBackend::CudaM2LP2P)
      .value("CUDA_PARTIAL", ExecutionBackend::CudaPartial)
      .value("CUDA_FULL", ExecutionBackend::CudaFull)
      .value("CUDA_M2L", ExecutionBackend::CudaM2L)
      .value("CUDA_M2L_STATIC_P2P", ExecutionBackend::CudaM2LStaticP2P)
      .value("CUDA_B200", ExecutionBackend::CudaB200);
  py::enum_<P2PExecutionPacking>(m, "P2PExecutionPacking")
      .value("REFERENCE", P2PExecutionPacking::Reference)
      .value("CANONICAL_AOS", P2PExecutionPacking::CanonicalAos)
      .value("PARTICLE_ROW_SOA", P2PExecutionPacking::ParticleRowSoa)
      .value("CUDA_BSR3", P2PExecutionPacking::CudaBsr3)
      .value("ON_THE_FLY", P2PExecutionPacking::OnTheFly);
  py::enum_<SourceGeometry>(m, "SourceGeometry")
      .value("POINT_DIPOLE", SourceGeometry::PointDipole)
      .value("UNIFORM_CUBOID", SourceGeometry::UniformCuboid);
  py::class_<CuboidSize>(m, "CuboidSize")
      .def(py::init([](double hx, double hy, double hz) { return CuboidSize{hx, hy, hz}; }), py::arg("hx"),
           py::arg("hy"), py::arg("hz"))
      .def_readwrite("hx", &CuboidSize::hx)
      .def_readwrite("hy", &CuboidSize::hy)
      .def_readwrite("hz", &CuboidSize::hz)
      .def_property_readonly("volume", [](const CuboidSize &h) { return h.hx * h.hy * h.hz; });
  py::enum_<StaticPrecision>(m, "StaticPrecision")
      .value("FLOAT32", StaticPrecision::Float32)
      .value("FLOAT64", StaticPrecision::Float64);
  py::enum_<B200M2L>(m, "B200M2L")
      .value("AUTO", B200M2L::Auto)
      .value("FLOAT32", B200M2L::Float32)
      .value("SPLIT_BF16", B200M2L::SplitBf16);

  m.def("cuda_compiled", &cuda_compiled);
  m.def("one_mkl_available", &one_mkl_available);
  m.def("cuda_available", &cuda_available);
  m.def("cuda_direct_available", &cuda_direct_available);
  m.def("cuda_m2l_p2p_available", &cuda_m2l_p2p_available);
  m.def("cuda_m2l_available", &cuda_m2l_available);
  m.def("cuda_full_available", &cuda_full_available);
  m.def("cuda_b200_available", &cuda_b200_available);
  m.def("cuda_device_description", &cuda_device_description);

  m.def("morton_encode", &morton_encode);
  m.def("morton_decode", &morton_decode);
  m.def("level_offset", &level_offset);
  m.def("node_index", &node_index);
  m.def("multi_indices", [](int order) {
    if (order < 0) throw std::invalid_argument("order must be non-negative");
    const MultiIndexSet b(order);
    std::vector<std::array<int, 3>> out;
    for (int i = 0; i < b.size(); ++i) out.push_back({b[i].ax, b[i].ay, b[i].az});
    return out;
  }, py::arg("order"));

  m.def(
      "cuda_direct_p2p_reference",
      [](py::object targets, py::object sources, py::object moments, const std::string &output, py::object ids) {
        const auto t = parse_vec3_array(targets, "target_positions");
        const auto s = parse_vec3_array(sources, "source_positions");
        const auto mo = parse_vec3_array(moments, "dipole_moments");
        if (s.size() != mo.size()) throw std::invalid_argument("sources and moments must contain the same number of rows");
        const OutputFlags flags = parse_output(output);
        std::vector<int> id = parse_ids(ids);
        if (!id.empty() && id.size() != t.size()) throw std::invalid_argument("identity map has incorrect length");
        std::vector<double> phi(t.size()), H(3 * t.size());
        int st;
        {
          py::gil_scoped_release release;
          st = cdfmm_b200_direct_fp64(0, static_cast<int32_t>(s.size()), reinterpret_cast<const double *>(s.data()),
                                      reinterpret_cast<const double *>(mo.data()), static_cast<int32_t>(t.size()),
                                      reinterpret_cast<const double *>(t.data()), id.empty() ? nullptr : id.data(),
                                      phi.data(), H.data());
        }
        if (st != CDFMM_B200_OK) {
          const std::string msg = cdfmm_b200_last_error(nullptr);
          if (st == CDFMM_B200_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
          throw std::runtime_error(msg);
        }
        py::array_t<double> aphi(static_cast<py::ssize_t>(t.size()));
        py::array_t<double> aH({static_cast<py::ssize_t>(t.size()), static_cast<py::ssize_t>(3)});
        auto p = aphi.mutable_unchecked<1>();
        auto h = aH.mutable_unchecked<2>();
        for (py::ssize_t i = 0; i < static_cast<py::ssize_t>(t.size()); ++i) {
          p(i) = has_flag(flags, OutputFlags::Potential) ? phi[static_cast<std::size_t>(i)] : 0.0;
          for (int c = 0; c < 3; ++c)
            h(i, c) = has_flag(flags, OutputFlags::Field) ? H[3 * static_cast<std::size_t>(i) + c] : 0.0;
        }
        py::dict d;
        d["phi"] = aphi;
        d["H"] = aH;
        return d;
      },
      py::arg("target_positions"), py::arg("source_positions"), py::arg("dipole_moments"),
      py::arg("output") = "field", py::arg("target_source_indices") = py::none(),
      "FP64 O(N*M) direct dipole sum on the CUDA device with explicit self exclusion.");

  py::class_<UniformFmmOptions>(m, "UniformFmmOptions")
      .def(py::init<>())
      .def_readwrite("precision", &UniformFmmOptions::precision)
      .def_readwrite("expansion_order", &UniformFmmOptions::expansion_order)
      .def_readwrite("tree", &UniformFmmOptions::tree)
      .def_readwrite("m2l_backend", &UniformFmmOptions::m2l_backend)
      .def_readwrite("static_matrix_backend", &UniformFmmOptions::static_matrix_backend)
      .def_readwrite("backend", &UniformFmmOptions::backend)
      .def_readwrite("source_geometry", &UniformFmmOptions::source_geometry)
      .def_readwrite("source_sizes", &UniformFmmOptions::source_sizes)
      .def_readwrite("use_cuboid_p2m", &UniformFmmOptions::use_cuboid_p2m)
      .def_readwrite("fixed_target_source_indices", &UniformFmmOptions::fixed_target_source_indices)
      .def_readwrite("cuda_p2p_bsr_max_bytes", &UniformFmmOptions::cuda_p2p_bsr_max_bytes)
      .def_readwrite("max_states", &UniformFmmOptions::max_states)
      .def_readwrite("b200_m2l", &UniformFmmOptions::b200_m2l)
      .def_readwrite("device", &UniformFmmOptions::device);

  py::class_<UniformFmm>(m, "UniformFmm")
      .def(py::init([](py::object s, const UniformFmmOptions &o) {
             return UniformFmm(parse_vec3_array(s, "source_positions"), o);
           }),
           py::arg("source_positions"), py::arg("options") = UniformFmmOptions{})
      .def(py::init([](py::object s, py::object t, const UniformFmmOptions &o) {
             return UniformFmm(parse_vec3_array(s, "source_positions"), parse_vec3_array(t, "target_positions"), o);
           }),
           py::arg("source_positions"), py::arg("target_positions"), py::arg("options") = UniformFmmOptions{})
      .def("upward_pass", [](UniformFmm &f, py::object mo) { f.upward_pass(parse_vec3_array(mo, "dipole_moments")); },
           py::arg("dipole_moments"))
      .def("downward_pass", &UniformFmm::downward_pass)
      .def(
          "evaluate",
          [](UniformFmm &f, py::object mo, const std::string &output, py::object ids) {
            const auto moments = parse_vec3_array(mo, "dipole_moments");
            const std::vector<int> id = parse_ids(ids);
            const OutputFlags flags = parse_output(output);
            std::vector<FloatPotentialField> r(f.tree().sorted_target_positions().size());
            {
              py::gil_scoped_release release;
              f.evaluate_into_float32(moments, r, flags, id);
            }
            return results_to_dict(r);
          },
          py::arg("dipole_moments"), py::arg("output") = "field", py::arg("target_source_indices") = py::none(),
          "Run the complete FMM and return values in target order.")
      .def(
          "evaluate_states",
          [](UniformFmm &f, py::object mo, const std::string &output, py::object ids) {
            const FloatArray a = py::cast<FloatArray>(mo);
            const py::ssize_t ns = static_cast<py::ssize_t>(f.tree().sorted_source_positions().size());
            if (a.ndim() != 3 || a.shape(1) != ns || a.shape(2) != 3)
              throw std::invalid_argument("dipole_moments must have shape (n_states, n_sources, 3)");
            const int K = static_cast<int>(a.shape(0));
            const py::ssize_t nt = static_cast<py::ssize_t>(f.tree().sorted_target_positions().size());
            const OutputFlags flags = parse_output(output);
            const std::vector<int> id = parse_ids(ids);
            py::array_t<float> H({static_cast<py::ssize_t>(K), nt, static_cast<py::ssize_t>(3)});
            py::array_t<float> phi({static_cast<py::ssize_t>(K), nt});
            std::fill(H.mutable_data(), H.mutable_data() + H.size(), 0.0F);
            std::fill(phi.mutable_data(), phi.mutable_data() + phi.size(), 0.0F);
            const bool want_h = has_flag(flags, OutputFlags::Field);
            const bool want_phi = has_flag(flags, OutputFlags::Potential);
            {
              py::gil_scoped_release release;
              f.evaluate_states_float32(std::span<const float>(a.data(), static_cast<std::size_t>(a.size())), K,
                                        want_h ? std::span<float>(H.mutable_data(), static_cast<std::size_t>(H.size()))
                                               : std::span<float>(),
                                        want_phi ? std::span<float>(phi.mutable_data(), static_cast<std::size_t>(phi.size()))
                                                 : std::span<float>(),
                                        flags, id);
            }
            py::dict d;
            d["phi"] = phi;
            d["H"] = H;
            return d;
          },
          py::arg("dipole_moments"), py::arg("output") = "field", py::arg("target_source_indices") = py::none(),
          "Evaluate K moment states (shape (K, n_sources, 3)) in one device call.")
      .def(
          "evaluate_device",
          [](UniformFmm &f, std::uintptr_t moments, int n_states, std::uintptr_t field, std::uintptr_t potential,
             const std::string &output, std::uintptr_t stream) {
            py::gil_scoped_release release;
            f.evaluate_device(reinterpret_cast<const float *>(moments), n_states, reinterpret_cast<float *>(field),
                              reinterpret_cast<float *>(potential), parse_output(output),
                              reinterpret_cast<void *>(stream));
          },
          py::arg("moments_ptr"), py::arg("n_states"), py::arg("field_ptr"), py::arg("potential_ptr") = 0,
          py::arg("output") = "field", py::arg("stream") = 0,
          "Evaluate K states on device-resident float32 arrays (device pointers), stream-ordered.")
      .def(
          "evaluate_into",
          [](UniformFmm &f, const py::object &moments, const py::object &field, const py::object &potential,
             const std::string &output, std::uintptr_t stream) {
            const OutputFlags flags = parse_output(output);
            const py::dict cai = moments.attr("__cuda_array_interface__");
            const py::tuple sh = cai["shape"];
            const long K = sh.size() == 3 ? sh[0].cast<long>() : 1;
            const long ns = static_cast<long>(f.tree().sorted_source_positions().size());
            const long nt = static_cast<long>(f.tree().sorted_target_positions().size());
            const std::uintptr_t m = cuda_array_ptr(moments, sh.size() == 3 ? std::vector<long>{K, ns, 3}
                                                                             : std::vector<long>{ns, 3}, "moments");
            std::uintptr_t h = 0, p = 0;
            if (has_flag(flags, OutputFlags::Field))
              h = cuda_array_ptr(field, sh.size() == 3 ? std::vector<long>{K, nt, 3} : std::vector<long>{nt, 3}, "field");
            if (has_flag(flags, OutputFlags::Potential))
              p = cuda_array_ptr(potential, sh.size() == 3 ? std::vector<long>{K, nt} : std::vector<long>{nt}, "potential");
            py::gil_scoped_release release;
            f.evaluate_device(reinterpret_cast<const float *>(m), static_cast<int>(K), reinterpret_cast<float *>(h),
                              reinterpret_cast<float *>(p), flags, reinterpret_cast<void *>(stream));
          },
          py::arg("dipole_moments"), py::arg("field") = py::none(), py::arg("potential") = py::none(),
          py::arg("output") = "field", py::arg("stream") = 0,
          "Zero-copy evaluation on CUDA arrays (torch tensors, ...): moments (K, n_sources, 3) or (n_sources, 3) "
          "float32 in user order; results written into `field` / `potential` in user order, stream-ordered.")
      .def_property_readonly("tree", &UniformFmm::tree, py::return_value_policy::reference_internal)
      .def_property_readonly("expansion_order", [](const UniformFmm &f) { return f.basis().order(); })
      .def_property_readonly("m2l_backend", &UniformFmm::m2l_backend)
      .def_property_readonly("backend", &UniformFmm::backend)
      .def_property_readonly("precision", &UniformFmm::precision)
      .def_property_readonly("p2p_execution_packing", &UniformFmm::p2p_execution_packing)
      .def_property_readonly("b200_m2l", &UniformFmm::b200_m2l)
      .def_property_readonly("max_states", &UniformFmm::max_states)
      .def_property_readonly("cuda_plan_statistics", [](const UniformFmm &f) {
        const CudaPlanStatistics &s = f.cuda_plan_statistics();
        py::dict d;
        d["scalar_bytes"] = s.scalar_bytes;
        d["m2m_unique_matrix_count"] = s.m2m_unique_matrix_count;
        d["m2m_matrix_bytes"] = s.m2m_matrix_bytes;
        d["m2l_unique_matrix_count"] = s.m2l_unique_matrix_count;
        d["m2l_matrix_bytes"] = s.m2l_matrix_bytes;
        d["m2l_interaction_metadata_bytes"] = s.m2l_interaction_metadata_bytes;
        d["l2l_unique_matrix_count"] = s.l2l_unique_matrix_count;
        d["l2l_matrix_bytes"] = s.l2l_matrix_bytes;
        d["setup_h2d_bytes"] = s.setup_h2d_bytes;
        d["evaluation_h2d_bytes"] = s.evaluation_h2d_bytes;
        d["evaluation_d2h_bytes"] = s.evaluation_d2h_bytes;
        d["evaluation_h2d_calls"] = s.evaluation_h2d_calls;
        d["evaluation_d2h_calls"] = s.evaluation_d2h_calls;
        d["persistent_device_bytes"] = s.persistent_device_bytes;
        d["p2p_tensor_bytes"] = s.p2p_tensor_bytes;
        d["p2p_index_bytes"] = s.p2p_index_bytes;
        d["p2p_row_metadata_bytes"] = s.p2p_row_metadata_bytes;
        d["p2p_leaf_metadata_bytes"] = s.p2p_leaf_metadata_bytes;
        d["p2p_identity_bytes"] = s.p2p_identity_bytes;
        d["p2p_scratch_bytes"] = s.p2p_scratch_bytes;
        d["p2p_threads_per_block"] = s.p2p_threads_per_block;
        d["plan_generation_count"] = s.plan_generation_count;
        d["static_upload_count"] = s.static_upload_count;
        d["static_m2l_upload_count"] = s.static_m2l_upload_count;
        d["m2l_interaction_count"] = s.m2l_interaction_count;
        d["p2p_interaction_count"] = s.p2p_interaction_count;
        return d;
      })
      .def_property_readonly("static_plan_statistics", [](const UniformFmm &f) {
        const StaticPlanStatistics &s = f.static_plan_statistics();
        py::dict d;
        d["scalar_bytes"] = s.scalar_bytes;
        d["transfer_classes"] = s.transfer_classes;
        d["interactions"] = s.interactions;
        d["operator_bytes"] = s.operator_bytes;
        d["interaction_bytes"] = s.interaction_bytes;
        d["scratch_bytes"] = s.scratch_bytes;
        d["state_bytes"] = s.state_bytes;
        d["m2m_operators"] = s.m2m_operators;
        d["m2m_theoretical_interactions"] = s.m2m_theoretical_interactions;
        d["m2m_operator_bytes"] = s.m2m_operator_bytes;
        d["m2l_operators"] = s.m2l_operators;
        d["m2l_theoretical_maximum_classes"] = StaticPlanStatistics::theoretical_maximum_m2l_classes;
        d["m2l_operator_bytes"] = s.m2l_operator_bytes;
        d["m2l_interaction_bytes"] = s.m2l_interaction_bytes;
        d["l2l_operators"] = s.l2l_operators;
        d["l2l_theoretical_interactions"] = s.l2l_theoretical_interactions;
        d["l2l_operator_bytes"] = s.l2l_operator_bytes;
        d["translation_operator_bytes"] = s.translation_operator_bytes();
        d["dense"] = s.dense;
        d["sparse"] = s.sparse;
        d["numerically_pruned"] = s.numerically_pruned;
        d["symmetry_compressed"] = s.symmetry_compressed;
        d["p2p_interactions"] = s.p2p_interactions;
        d["total_bytes"] = s.total_bytes();
        d["setup_seconds"] = s.total.total_seconds;
        return d;
      })
      .def_property_readonly("last_timings", [](const UniformFmm &f) {
        const EvaluationTimings &t = f.last_timings();
        py::dict d;
        d["moment_permutation"] = phase(t.moment_permutation);
        d["p2m"] = phase(t.p2m);
        d["m2m"] = phase(t.m2m);
        d["m2l"] = phase(t.m2l);
        d["l2l"] = phase(t.l2l);
        d["l2p"] = phase(t.l2p);
        d["p2p"] = phase(t.p2p);
        d["cuda_kernel"] = phase(t.cuda_kernel);
        d["total"] = phase(t.total);
        d["evaluations"] = t.evaluations;
        return d;
      })
      .def("set_stage_timing", [](UniformFmm &f, bool on) { cdfmm_b200_set_timing(f.device_plan(), on ? 1 : 0); },
           py::arg("enabled"), "Record per-stage CUDA-event times into last_timings.")
      .def_property_readonly("root_multipole", [](const UniformFmm &f) { return floats_to_array(f.root_multipole_float32()); })
      .def("multipole", [](const UniformFmm &f, int i) { return floats_to_array(f.multipole_float32(i)); },
           py::arg("node_index"))
      .def("local", [](const UniformFmm &f, int i) { return floats_to_array(f.local_float32(i)); }, py::arg("node_index"))
      .def_property_readonly("device_plan_address", [](const UniformFmm &f) {
        return reinterpret_cast<std::uintptr_t>(f.device_plan());
      });
}
