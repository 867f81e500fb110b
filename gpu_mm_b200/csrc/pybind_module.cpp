// pybind11 module gpu_mm_pybind11: the reference's Python binding surface
// (kmsmith137/gpu_mm src_pybind11/gpu_mm_pybind11.cu:77-193) over this library's C++ API.
//
// Arrays are accepted from any object exposing __cuda_array_interface__ (torch CUDA tensors, cupy)
// or __array_interface__ (numpy), and from torch CPU tensors; float32 only for maps, TODs and
// xpointing, like the reference's Tmm = float.  GPU work runs with the GIL released.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <cstring>
#include <string>

#include "../../include/gpu_mm_b200/gpu_mm.hpp"

namespace py = pybind11;
using namespace gpu_mm;

namespace {

template<typename T> struct TypeCodes;
template<> struct TypeCodes<float> { static bool ok(const std::string &t) { return t == "<f4" || t == "=f4"; } };
template<> struct TypeCodes<double> { static bool ok(const std::string &t) { return t == "<f8" || t == "=f8"; } };
template<> struct TypeCodes<int> { static bool ok(const std::string &t) { return t == "<i4" || t == "=i4"; } };
template<> struct TypeCodes<long> { static bool ok(const std::string &t) { return t == "<i8" || t == "=i8"; } };
template<> struct TypeCodes<uint> {
    static bool ok(const std::string &t) { return t == "<u4" || t == "<i4" || t == "=u4" || t == "=i4"; }
};
template<> struct TypeCodes<ulong> {
    static bool ok(const std::string &t) { return t == "<u8" || t == "<i8" || t == "=u8" || t == "=i8"; }
};
template<> struct TypeCodes<unsigned char> {
    static bool ok(const std::string &t) { return t == "|u1" || t == "|i1" || t == "<u1" || t == "|b1"; }
};

std::shared_ptr<void> keep_alive(py::object obj)
{
    auto *held = new py::object(std::move(obj));
    return std::shared_ptr<void>(held, [](void *p) {
        py::gil_scoped_acquire gil;
        delete (py::object *) p;
    });
}

template<typename T>
Array<T> to_array(py::handle h, const char *name)
{
    py::object obj = py::reinterpret_borrow<py::object>(h);
    py::dict d;
    bool gpu = false;
    if (py::hasattr(obj, "__cuda_array_interface__")) {
        d = obj.attr("__cuda_array_interface__");
        gpu = true;
    } else if (py::hasattr(obj, "__array_interface__")) {
        d = obj.attr("__array_interface__");
    } else if (py::hasattr(obj, "numpy") && py::hasattr(obj, "is_cuda") && !obj.attr("is_cuda").cast<bool>()) {
        obj = obj.attr("detach")().attr("numpy")();
        d = obj.attr("__array_interface__");
    } else {
        throw std::runtime_error(std::string("gpu_mm: argument '") + name + "' is not an array");
    }
    const std::string typestr = d["typestr"].cast<std::string>();
    if (!TypeCodes<T>::ok(typestr))
        throw std::runtime_error(std::string("gpu_mm: argument '") + name + "' has unsupported dtype " + typestr);
    py::tuple data = d["data"];
    T *ptr = reinterpret_cast<T *>(data[0].cast<uintptr_t>());
    py::tuple shape_t = d["shape"];
    std::vector<long> shape;
    for (auto s : shape_t)
        shape.push_back(s.cast<long>());
    if (shape.empty())
        shape.push_back(1);
    if (shape.size() > 4)
        throw std::runtime_error(std::string("gpu_mm: argument '") + name + "' has more than 4 dimensions");
    std::vector<long> strides;
    if (d.contains("strides") && !d["strides"].is_none()) {
        py::tuple st = d["strides"];
        for (auto s : st) {
            long b = s.cast<long>();
            if (b % (long) sizeof(T))
                throw std::runtime_error(std::string("gpu_mm: argument '") + name + "' has unaligned strides");
            strides.push_back(b / (long) sizeof(T));
        }
        if (strides.size() != shape.size())
            strides.clear();
    }
    if (strides.empty()) {
        strides.assign(shape.size(), 1);
        for (int i = (int) shape.size() - 2; i >= 0; i--)
            strides[i] = strides[i + 1] * shape[i + 1];
    }
    return Array<T>(ptr, shape, strides, gpu, keep_alive(obj));
}

template<typename T>
py::array_t<T> host_to_numpy(const Array<T> &a)
{
    py::array_t<T> ret(a.size);
    std::memcpy(ret.mutable_data(), a.data, a.size * sizeof(T));
    return ret;
}

}  // namespace

PYBIND11_MODULE(gpu_mm_pybind11, m)
{
    m.doc() = "gpu_mm_b200: B200-native pointing operators (drop-in for gpu_mm.gpu_mm_pybind11)";

    m.def("_get_tsize", []() { return sizeof(float); });
    // ---- Batches of TODs (raw device pointers; gpu_mm_b200.batch.TodBatch wraps them) ----
    auto tuning_of = [](py::object t) {
        gmm_batch_tuning bt;
        throw_on_error(gmm_batch_tuning_default(&bt));
        if (!t.is_none()) {
            py::tuple tt = t.cast<py::tuple>();
            bt.sort_digit_bits = tt[0].cast<int>();
            bt.ctas_per_sm = tt[1].cast<int>();
            bt.min_lines_per_cta = tt[2].cast<int>();
        }
        return bt;
    };
    m.def("batch_tuning_default", []() {
        gmm_batch_tuning bt;
        throw_on_error(gmm_batch_tuning_default(&bt));
        return py::make_tuple(bt.sort_digit_bits, bt.ctas_per_sm, bt.min_lines_per_cta);
    });
    m.def("batch_plan_nbytes", [tuning_of](long total_lines, int ny, int nx, py::object tuning) {
        gmm_batch_tuning bt = tuning_of(tuning);
        int64_t pn = 0, tn = 0;
        throw_on_error(gmm_batch_plan_nbytes(total_lines, ny, nx, &bt, &pn, &tn));
        return py::make_tuple(pn, tn);
    }, py::arg("total_lines"), py::arg("nypix_global"), py::arg("nxpix_global"), py::arg("tuning") = py::none());
    m.def("batch_plan_build",
          [tuning_of](uintptr_t descs, int ntod, long total_lines, int ny, int nx, bool periodic, uintptr_t plan,
                      long plan_nbytes, uintptr_t tmp, long tmp_nbytes, py::object tuning, uintptr_t errword,
                      uintptr_t stream) {
              gmm_batch_tuning bt = tuning_of(tuning);
              py::gil_scoped_release rel;
              throw_on_error(gmm_batch_plan_build((const gmm_tod_desc *) descs, ntod, total_lines, ny, nx, periodic,
                                                  (void *) plan, plan_nbytes, (void *) tmp, tmp_nbytes, &bt,
                                                  (uint32_t *) errword, (cudaStream_t) stream));
          },
          py::arg("descs"), py::arg("ntod"), py::arg("total_lines"), py::arg("nypix_global"), py::arg("nxpix_global"),
          py::arg("periodic_xcoord"), py::arg("plan"), py::arg("plan_nbytes"), py::arg("tmp"), py::arg("tmp_nbytes"),
          py::arg("tuning"), py::arg("errword"), py::arg("stream") = 0);
    m.def("batch_plan_each_tmp_nbytes", [tuning_of](long total_lines, int ntod, int ny, int nx, py::object tuning) {
        gmm_batch_tuning bt = tuning_of(tuning);
        int64_t tn = 0;
        throw_on_error(gmm_batch_plan_each_tmp_nbytes(total_lines, ntod, ny, nx, &bt, &tn));
        return tn;
    }, py::arg("total_lines"), py::arg("ntod"), py::arg("nypix_global"), py::arg("nxpix_global"),
       py::arg("tuning") = py::none());
    m.def("batch_plan_build_each",
          [tuning_of](uintptr_t descs, int ntod, long total_lines, int ny, int nx, bool periodic, uintptr_t plans,
                      uintptr_t tmp, long tmp_nbytes, py::object tuning, uintptr_t errword, uintptr_t stream) {
              gmm_batch_tuning bt = tuning_of(tuning);
              py::gil_scoped_release rel;
              throw_on_error(gmm_batch_plan_build_each((const gmm_tod_desc *) descs, ntod, total_lines, ny, nx,
                                                       periodic, (void *const *) plans, (void *) tmp, tmp_nbytes, &bt,
                                                       (uint32_t *) errword, (cudaStream_t) stream));
          },
          py::arg("descs"), py::arg("ntod"), py::arg("total_lines"), py::arg("nypix_global"), py::arg("nxpix_global"),
          py::arg("periodic_xcoord"), py::arg("plans"), py::arg("tmp"), py::arg("tmp_nbytes"), py::arg("tuning"),
          py::arg("errword"), py::arg("stream") = 0);
    m.def("batch_plan_merge",
          [tuning_of](uintptr_t plans, uintptr_t nlines, int ntod, long total_lines, int ny, int nx, uintptr_t plan,
                      long plan_nbytes, uintptr_t tmp, long tmp_nbytes, py::object tuning, uintptr_t stream) {
              gmm_batch_tuning bt = tuning_of(tuning);
              py::gil_scoped_release rel;
              throw_on_error(gmm_batch_plan_merge((const void *const *) plans, (const int64_t *) nlines, ntod,
                                                  total_lines, ny, nx, (void *) plan, plan_nbytes, (void *) tmp,
                                                  tmp_nbytes, &bt, (cudaStream_t) stream));
          },
          py::arg("plans"), py::arg("nlines"), py::arg("ntod"), py::arg("total_lines"), py::arg("nypix_global"),
          py::arg("nxpix_global"), py::arg("plan"), py::arg("plan_nbytes"), py::arg("tmp"), py::arg("tmp_nbytes"),
          py::arg("tuning"), py::arg("stream") = 0);
    m.def("batch_map2tod",
          [tuning_of](uintptr_t descs, int ntod, long total_lines, py::object local_map, const LocalPixelization &lpix,
                      uintptr_t plan, bool partial_pixelization, bool accum, py::object tuning, uintptr_t errword,
                      uintptr_t stream) {
              Array<float> m_ = to_array<float>(local_map, "local_map");
              if (!m_.gpu || m_.size != 3 * lpix.npix)
                  throw std::runtime_error("batch_map2tod: local_map must be a GPU array of size 3*npix");
              gmm_batch_tuning bt = tuning_of(tuning);
              gmm_lpix v = lpix.device_view();
              py::gil_scoped_release rel;
              throw_on_error(gmm_batch_map2tod((const gmm_tod_desc *) descs, ntod, total_lines, m_.data, &v,
                                               (const void *) plan, partial_pixelization, accum, &bt,
                                               (uint32_t *) errword, (cudaStream_t) stream));
          },
          py::arg("descs"), py::arg("ntod"), py::arg("total_lines"), py::arg("local_map"), py::arg("local_pixelization"),
          py::arg("plan"), py::arg("partial_pixelization"), py::arg("accum"), py::arg("tuning"), py::arg("errword"),
          py::arg("stream") = 0);
    m.def("batch_tod2map",
          [tuning_of](uintptr_t descs, int ntod, long total_lines, py::object local_map, const LocalPixelization &lpix,
                      uintptr_t plan, bool partial_pixelization, py::object tuning, uintptr_t errword,
                      uintptr_t stream) {
              Array<float> m_ = to_array<float>(local_map, "local_map");
              if (!m_.gpu || m_.size != 3 * lpix.npix)
                  throw std::runtime_error("batch_tod2map: local_map must be a GPU array of size 3*npix");
              gmm_batch_tuning bt = tuning_of(tuning);
              gmm_lpix v = lpix.device_view();
              py::gil_scoped_release rel;
              throw_on_error(gmm_batch_tod2map((const gmm_tod_desc *) descs, ntod, total_lines, m_.data, &v,
                                               (const void *) plan, partial_pixelization, &bt, (uint32_t *) errword,
                                               (cudaStream_t) stream));
          },
          py::arg("descs"), py::arg("ntod"), py::arg("total_lines"), py::arg("local_map"), py::arg("local_pixelization"),
          py::arg("plan"), py::arg("partial_pixelization"), py::arg("tuning"), py::arg("errword"),
          py::arg("stream") = 0);
    m.def("errword_read", [](uintptr_t errword, unsigned ignore, uintptr_t stream) {
        py::gil_scoped_release rel;
        throw_on_error(gmm_errword_read((const uint32_t *) errword, ignore, (cudaStream_t) stream));
    }, py::arg("errword"), py::arg("ignore") = 0, py::arg("stream") = 0);

    m.def("_version", []() { return std::string(gmm_version()); });
    m.def("_set_sort_digit_bits", [](int bits) { throw_on_error(gmm_set_sort_digit_bits(bits)); });
    m.def("_get_sort_digit_bits", []() { return gmm_get_sort_digit_bits(); });

    py::class_<LocalPixelization>(m, "LocalPixelization",
                                  "LocalPixelization: represents a set of map cells, held on a single GPU")
        .def(py::init([](long nypix_global, long nxpix_global, py::object cell_offsets_cpu, py::object cell_offset_gpu,
                         long ystride, long polstride, bool periodic_xcoord) {
                 return new LocalPixelization(nypix_global, nxpix_global, to_array<long>(cell_offsets_cpu, "cell_offsets_cpu"),
                                              to_array<long>(cell_offset_gpu, "cell_offset_gpu"), ystride, polstride,
                                              periodic_xcoord);
             }),
             py::arg("nypix_global"), py::arg("nxpix_global"), py::arg("cell_offsets_cpu"), py::arg("cell_offset_gpu"),
             py::arg("ystride"), py::arg("polstride"), py::arg("periodic_xcoord"))
        .def_readonly("nypix_global", &LocalPixelization::nypix_global)
        .def_readonly("nxpix_global", &LocalPixelization::nxpix_global)
        .def_readonly("periodic_xcoord", &LocalPixelization::periodic_xcoord)
        .def_readonly("ystride", &LocalPixelization::ystride)
        .def_readonly("polstride", &LocalPixelization::polstride)
        .def_readonly("nycells", &LocalPixelization::nycells)
        .def_readonly("nxcells", &LocalPixelization::nxcells)
        .def_readwrite("npix", &LocalPixelization::npix, "counts only local pixels, does not include factor 3 from TQU.")
        .def("copy_gpu_offsets_to_cpu", &LocalPixelization::copy_gpu_offsets_to_cpu)
        .def("copy_cpu_offsets_to_gpu", &LocalPixelization::copy_cpu_offsets_to_gpu);

    py::class_<PointingPrePlan>(m, "PointingPrePlan",
                                "PointingPrePlan(xpointing_gpu, nypix_global, nxpix_global)\n\n"
                                "Plan creation is factored into two steps: a small PointingPrePlan (a few KB),\n"
                                "then a PointingPlan (~100 MB) built from it and the xpointing array.")
        .def(py::init([](py::object xpointing_gpu, long nypix_global, long nxpix_global, py::object nmt_gpu,
                         py::object err_gpu, bool periodic_xcoord, bool debug) {
                 Array<float> xp = to_array<float>(xpointing_gpu, "xpointing_gpu");
                 Array<uint> nmt = to_array<uint>(nmt_gpu, "nmt_gpu");
                 Array<uint> err = to_array<uint>(err_gpu, "err_gpu");
                 py::gil_scoped_release rel;
                 return new PointingPrePlan(xp, nypix_global, nxpix_global, nmt, err, periodic_xcoord, debug);
             }),
             py::arg("xpointing_gpu"), py::arg("nypix_global"), py::arg("nxpix_global"), py::arg("nmt_gpu"),
             py::arg("err_gpu"), py::arg("periodic_xcoord"), py::arg("debug"))
        .def_static("_get_preplan_size", []() { return PointingPrePlan::preplan_size; })
        .def_readonly("nsamp", &PointingPrePlan::nsamp, "Number of TOD samples")
        .def_readonly("nypix_global", &PointingPrePlan::nypix_global, "Number of y-pixels")
        .def_readonly("nxpix_global", &PointingPrePlan::nxpix_global, "Number of x-pixels")
        .def_readonly("periodic_xcoord", &PointingPrePlan::periodic_xcoord, "Boolean flag, indicates whether x-coordinate is periodic")
        .def_readonly("plan_nbytes", &PointingPrePlan::plan_nbytes, "Length of 'buf' argument to PointingPlan constructor")
        .def_readonly("plan_constructor_tmp_nbytes", &PointingPrePlan::plan_constructor_tmp_nbytes,
                      "Length of 'tmp_buf' argument to PointingPlan constructor")
        .def_readonly("overhead", &PointingPrePlan::overhead, "typically ~0.3 (meaning that cell decomposition is a ~30% overhead)")
        .def_readonly("ncl_per_threadblock", &PointingPrePlan::ncl_per_threadblock, "Used when launching planner/preplanner kernels")
        .def_readonly("planner_nblocks", &PointingPrePlan::planner_nblocks, "Used when launching planner/preplanner kernels")
        .def_readonly("nmt_per_threadblock", &PointingPrePlan::nmt_per_threadblock, "Used in pointing operations (map2tod/tod2map)")
        .def_readonly("pointing_nblocks", &PointingPrePlan::pointing_nblocks, "Used in pointing operations (map2tod/tod2map)")
        .def_readonly("plan_nmt", &PointingPrePlan::plan_nmt, "Total number of mt-pairs in plan")
        .def_readonly("cub_nbytes", &PointingPrePlan::cub_nbytes, "Number of bytes of radix-sort scratch in 'tmp_buf'")
        .def_property_readonly("sort_digit_bits", [](const PointingPrePlan &p) { return p.info.sort_digit_bits; })
        .def("get_nmt_cumsum", [](const PointingPrePlan &p) { return host_to_numpy(p.get_nmt_cumsum()); },
             "Copies nmt_cumsum array to host, and returns it as a numpy array.")
        .def("__str__", &PointingPrePlan::str);

    py::class_<PointingPlan>(m, "PointingPlan", "PointingPlan(preplan, xpointing_gpu)")
        .def(py::init([](const PointingPrePlan &preplan, py::object xpointing_gpu, py::object buf, py::object tmp_buf,
                         bool debug) {
                 Array<float> xp = to_array<float>(xpointing_gpu, "xpointing_gpu");
                 Array<unsigned char> b = to_array<unsigned char>(buf, "buf");
                 Array<unsigned char> t = to_array<unsigned char>(tmp_buf, "tmp_buf");
                 py::gil_scoped_release rel;
                 return new PointingPlan(preplan, xp, b, t, debug);
             }),
             py::arg("preplan"), py::arg("xpointing_gpu"), py::arg("buf"), py::arg("tmp_buf"), py::arg("debug") = false)
        .def_readonly("nsamp", &PointingPlan::nsamp, "Number of TOD samples")
        .def_readonly("nypix_global", &PointingPlan::nypix_global, "Number of y-pixels")
        .def_readonly("nxpix_global", &PointingPlan::nxpix_global, "Number of x-pixels")
        .def_readonly("periodic_xcoord", &PointingPlan::periodic_xcoord, "Boolean flag, indicates whether x-coordinate is periodic")
        .def_property_readonly("plan_nmt", [](const PointingPlan &p) { return p.pp.plan_nmt; })
        .def_property_readonly("_buf_ptr", [](const PointingPlan &p) { return (uintptr_t) p.buf.data; })
        .def_property_readonly("_plan_mt_ptr", [](const PointingPlan &p) { return (uintptr_t) p.plan_mt; })
        .def_property_readonly("_owner_mt_ptr", [](const PointingPlan &p) { return (uintptr_t) p.owner_mt; })
        .def("_check_errflags", &PointingPlan::_check_errflags, py::arg("where"))
        .def("get_plan_mt", [](const PointingPlan &p) { return host_to_numpy(p.get_plan_mt(false)); },
             "Length nmt_cumsum[-1] array, sorted by (map cell, cache line)")
        .def("_get_owner_mt", [](const PointingPlan &p) { return host_to_numpy(p.get_owner_mt(false)); },
             "One word per cache line (cell | line << 20 | mflag << 46 | row band << 48), sorted by "
             "(the line's lowest cell, row band, line)")
        .def("_get_band_words", [](const PointingPlan &p) { return host_to_numpy(p.get_band_words(false)); },
             "One word per owner entry: the line's shape for the tod2map band path (0: not on that path)")
        .def("__str__", &PointingPlan::str);

    // Test utilities (gpu_mm_pybind11.cu:228-262).  ToyPointing fills caller-allocated arrays.
    py::class_<ToyPointing<float>>(m, "ToyPointing")
        .def(py::init([](long nypix_global, long nxpix_global, double scan_speed, double total_drift,
                         py::object xpointing_cpu, py::object xpointing_gpu, bool noisy) {
                 Array<float> c = to_array<float>(xpointing_cpu, "xpointing_cpu");
                 Array<float> g = to_array<float>(xpointing_gpu, "xpointing_gpu");
                 return new ToyPointing<float>(nypix_global, nxpix_global, scan_speed, total_drift, c, g, noisy);
             }),
             py::arg("nypix_global"), py::arg("nxpix_global"), py::arg("scan_speed"), py::arg("total_drift"),
             py::arg("xpointing_cpu"), py::arg("xpointing_gpu"), py::arg("noisy"))
        .def_readonly("nypix_global", &ToyPointing<float>::nypix_global, "Number of y-pixels")
        .def_readonly("nxpix_global", &ToyPointing<float>::nxpix_global, "Number of x-pixels")
        .def_readonly("scan_speed", &ToyPointing<float>::scan_speed, "Scan speed in map pixels per TOD sample")
        .def_readonly("total_drift", &ToyPointing<float>::total_drift, "Total drift over full TOD, in x-pixels")
        .def_readonly("drift_speed", &ToyPointing<float>::drift_speed, "Drift (in x-pixels) per TOD sample")
        .def("__str__", &ToyPointing<float>::str);

    py::class_<PointingPlanTester>(m, "PointingPlanTester", "PointingPlanTester: A utility class used in unit tests")
        .def(py::init([](const PointingPrePlan &preplan, py::object xpointing_gpu, py::object tmp) {
                 Array<float> xp = to_array<float>(xpointing_gpu, "xpointing_gpu");
                 Array<unsigned char> t = to_array<unsigned char>(tmp, "tmp");
                 py::gil_scoped_release rel;
                 return new PointingPlanTester(preplan, xp, t);
             }),
             py::arg("preplan"), py::arg("xpointing_gpu"), py::arg("tmp"))
        .def_readonly("nsamp", &PointingPlanTester::nsamp, "Number of TOD samples")
        .def_readonly("nypix_global", &PointingPlanTester::nypix_global, "Number of y-pixels")
        .def_readonly("nxpix_global", &PointingPlanTester::nxpix_global, "Number of x-pixels")
        .def_readonly("plan_nmt", &PointingPlanTester::plan_nmt, "Total number of mt-pairs in plan")
        .def_readonly("ncl_per_threadblock", &PointingPlanTester::ncl_per_threadblock, "Used when launching planner/preplanner kernels")
        .def_readonly("planner_nblocks", &PointingPlanTester::planner_nblocks, "Used when launching planner/preplanner kernels")
        .def_property_readonly("iypix", [](const PointingPlanTester &p) { return host_to_numpy(p.iypix_arr); },
                               "Length-nsamp array containing integer y-pixel indices")
        .def_property_readonly("ixpix", [](const PointingPlanTester &p) { return host_to_numpy(p.ixpix_arr); },
                               "Length-nsamp array containing integer x-pixel indices")
        .def_property_readonly("nmt_cumsum", [](const PointingPlanTester &p) { return host_to_numpy(p.nmt_cumsum); },
                               "Length-nblocks array containing integer cumulative counts")
        .def_property_readonly("sorted_mt", [](const PointingPlanTester &p) { return host_to_numpy(p.sorted_mt); },
                               "Length nmt_cumsum[-1], see PointingPlan docstring for 'mt' format")
        .def_static("get_constructor_tmp_nbytes", &PointingPlanTester::get_constructor_tmp_nbytes, py::arg("preplan"))
        .def("__str__", &PointingPlanTester::str);

    m.def("planned_map2tod",
          [](py::object tod, py::object local_map, py::object xpointing, const LocalPixelization &lpix,
             const PointingPlan &plan, bool partial_pixelization, bool debug, bool accum) {
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              py::gil_scoped_release rel;
              launch_planned_map2tod<float>(t, m_, x, lpix, plan, partial_pixelization, debug, accum);
          },
          py::arg("tod"), py::arg("local_map"), py::arg("xpointing"), py::arg("local_pixelization"), py::arg("plan"),
          py::arg("partial_pixelization"), py::arg("debug"), py::arg("accum"));

    // Precision variants of planned tod2map (no counterpart in the reference).
    m.def("planned_tod2map_compensated",
          [](py::object local_map, py::object comp, py::object tod, py::object xpointing,
             const LocalPixelization &lpix, const PointingPlan &plan, bool partial_pixelization, long max_run_lines) {
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> c = to_array<float>(comp, "comp");
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              py::gil_scoped_release rel;
              launch_planned_tod2map_compensated(m_, c, t, x, lpix, plan, partial_pixelization, max_run_lines);
          },
          py::arg("local_map"), py::arg("comp"), py::arg("tod"), py::arg("xpointing"), py::arg("local_pixelization"),
          py::arg("plan"), py::arg("partial_pixelization") = false, py::arg("max_run_lines") = 0);

    m.def("planned_tod2map_f64",
          [](py::object local_map, py::object tod, py::object xpointing, const LocalPixelization &lpix,
             const PointingPlan &plan, bool partial_pixelization, long max_run_lines) {
              Array<double> m_ = to_array<double>(local_map, "local_map");
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              py::gil_scoped_release rel;
              launch_planned_tod2map_f64(m_, t, x, lpix, plan, partial_pixelization, max_run_lines);
          },
          py::arg("local_map"), py::arg("tod"), py::arg("xpointing"), py::arg("local_pixelization"), py::arg("plan"),
          py::arg("partial_pixelization") = false, py::arg("max_run_lines") = 0);

    // float64 only for high-hit cells (no counterpart in the reference).
    py::class_<HotCells>(m, "HotCells",
                         "Cells of a LocalPixelization whose tod2map partials are reduced in float64 "
                         "(planned_tod2map_hot_f64), chosen by the cache lines of the given plans touching them")
        .def(py::init([](const LocalPixelization &lpix, py::list plans, long min_lines) {
                 std::vector<const PointingPlan *> v;
                 for (py::handle h : plans)
                     v.push_back(&h.cast<const PointingPlan &>());
                 py::gil_scoped_release rel;
                 return new HotCells(lpix, v, min_lines);
             }),
             py::arg("local_pixelization"), py::arg("plans"), py::arg("min_lines"), py::keep_alive<1, 2>())
        .def_readonly("min_lines", &HotCells::min_lines, "Cache lines a cell needs to be hot")
        .def_readonly("nhot", &HotCells::nhot, "Number of hot cells")
        .def("get_lines", [](const HotCells &h) { return host_to_numpy(h.get_lines()); },
             "Cache lines of the plans touching each cell (flat, iycell * nxcells + ixcell)")
        .def("get_slot", [](const HotCells &h) { return host_to_numpy(h.get_slot()); },
             "Accumulator slot of each cell, -1 if the cell is not hot (flat, iycell * nxcells + ixcell)")
        .def("fold",
             [](HotCells &h, py::object local_map, const LocalPixelization &lpix) {
                 Array<float> m_ = to_array<float>(local_map, "local_map");
                 py::gil_scoped_release rel;
                 h.fold(m_, lpix);
             },
             py::arg("local_map"), py::arg("local_pixelization"),
             "Adds the float64 accumulators into the float local map (one rounding per value) and zeroes them");

    m.def("planned_tod2map_hot_f64",
          [](py::object local_map, HotCells &hot, py::object tod, py::object xpointing, const LocalPixelization &lpix,
             const PointingPlan &plan, bool partial_pixelization, long max_run_lines) {
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              py::gil_scoped_release rel;
              launch_planned_tod2map_hot_f64(m_, hot, t, x, lpix, plan, partial_pixelization, max_run_lines);
          },
          py::arg("local_map"), py::arg("hot"), py::arg("tod"), py::arg("xpointing"), py::arg("local_pixelization"),
          py::arg("plan"), py::arg("partial_pixelization") = false, py::arg("max_run_lines") = 0);

    m.def("fold_compensation",
          [](py::object local_map, py::object comp) {
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> c = to_array<float>(comp, "comp");
              py::gil_scoped_release rel;
              fold_compensation(m_, c);
          },
          py::arg("local_map"), py::arg("comp"));

    m.def("planned_tod2map",
          [](py::object local_map, py::object tod, py::object xpointing, const LocalPixelization &lpix,
             const PointingPlan &plan, bool partial_pixelization, bool debug) {
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              py::gil_scoped_release rel;
              launch_planned_tod2map<float>(m_, t, x, lpix, plan, partial_pixelization, debug);
          },
          py::arg("local_map"), py::arg("tod"), py::arg("xpointing"), py::arg("local_pixelization"), py::arg("plan"),
          py::arg("partial_pixelization"), py::arg("debug"));

    m.def("response_map2tod",
          [](py::object tod, py::object local_map, py::object xpointing, py::object response,
             const LocalPixelization &lpix, const PointingPlan &plan, bool partial_pixelization, bool debug, bool accum) {
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              Array<float> r = to_array<float>(response, "response");
              py::gil_scoped_release rel;
              launch_response_map2tod<float>(t, m_, x, r, lpix, plan, partial_pixelization, debug, accum);
          },
          py::arg("tod"), py::arg("local_map"), py::arg("xpointing"), py::arg("response"),
          py::arg("local_pixelization"), py::arg("plan"), py::arg("partial_pixelization"), py::arg("debug"),
          py::arg("accum"));

    m.def("response_tod2map",
          [](py::object local_map, py::object tod, py::object xpointing, py::object response,
             const LocalPixelization &lpix, const PointingPlan &plan, bool partial_pixelization, bool debug) {
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              Array<float> r = to_array<float>(response, "response");
              py::gil_scoped_release rel;
              launch_response_tod2map<float>(m_, t, x, r, lpix, plan, partial_pixelization, debug);
          },
          py::arg("local_map"), py::arg("tod"), py::arg("xpointing"), py::arg("response"),
          py::arg("local_pixelization"), py::arg("plan"), py::arg("partial_pixelization"), py::arg("debug"));

    m.def("unplanned_map2tod",
          [](py::object tod, py::object local_map, py::object xpointing, const LocalPixelization &lpix,
             py::object errflags, bool partial_pixelization, bool accum) {
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              Array<uint> e = to_array<uint>(errflags, "errflags");
              py::gil_scoped_release rel;
              launch_unplanned_map2tod<float>(t, m_, x, lpix, e, partial_pixelization, accum);
          },
          py::arg("tod"), py::arg("local_map"), py::arg("xpointing"), py::arg("local_pixelization"),
          py::arg("errflags"), py::arg("partial_pixelization"), py::arg("accum"));

    m.def("unplanned_tod2map",
          [](py::object local_map, py::object tod, py::object xpointing, const LocalPixelization &lpix,
             py::object errflags, bool partial_pixelization) {
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              Array<uint> e = to_array<uint>(errflags, "errflags");
              py::gil_scoped_release rel;
              launch_unplanned_tod2map<float>(m_, t, x, lpix, e, partial_pixelization);
          },
          py::arg("local_map"), py::arg("tod"), py::arg("xpointing"), py::arg("local_pixelization"),
          py::arg("errflags"), py::arg("partial_pixelization"));

    // Non-blocking forms (deferred error check): errword is a 1-element 32-bit device array, stream a
    // CUDA stream handle (e.g. torch.cuda.current_stream().cuda_stream; 0 = legacy default stream).
    m.def("planned_map2tod_async",
          [](py::object tod, py::object local_map, py::object xpointing, const LocalPixelization &lpix,
             const PointingPlan &plan, bool partial_pixelization, bool accum, py::object errword, uintptr_t stream) {
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              Array<uint> e = to_array<uint>(errword, "errword");
              py::gil_scoped_release rel;
              launch_planned_map2tod_async(t, m_, x, lpix, plan, partial_pixelization, accum, e.data,
                                           (cudaStream_t) stream);
          },
          py::arg("tod"), py::arg("local_map"), py::arg("xpointing"), py::arg("local_pixelization"), py::arg("plan"),
          py::arg("partial_pixelization"), py::arg("accum"), py::arg("errword"), py::arg("stream") = 0);

    m.def("planned_tod2map_async",
          [](py::object local_map, py::object tod, py::object xpointing, const LocalPixelization &lpix,
             const PointingPlan &plan, bool partial_pixelization, py::object errword, uintptr_t stream) {
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              Array<uint> e = to_array<uint>(errword, "errword");
              py::gil_scoped_release rel;
              launch_planned_tod2map_async(m_, t, x, lpix, plan, partial_pixelization, e.data, (cudaStream_t) stream);
          },
          py::arg("local_map"), py::arg("tod"), py::arg("xpointing"), py::arg("local_pixelization"), py::arg("plan"),
          py::arg("partial_pixelization"), py::arg("errword"), py::arg("stream") = 0);

    m.def("unplanned_map2tod_async",
          [](py::object tod, py::object local_map, py::object xpointing, const LocalPixelization &lpix,
             bool partial_pixelization, bool accum, py::object errword, uintptr_t stream) {
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              Array<uint> e = to_array<uint>(errword, "errword");
              py::gil_scoped_release rel;
              launch_unplanned_map2tod_async(t, m_, x, lpix, partial_pixelization, accum, e.data, (cudaStream_t) stream);
          },
          py::arg("tod"), py::arg("local_map"), py::arg("xpointing"), py::arg("local_pixelization"),
          py::arg("partial_pixelization"), py::arg("accum"), py::arg("errword"), py::arg("stream") = 0);

    m.def("unplanned_tod2map_async",
          [](py::object local_map, py::object tod, py::object xpointing, const LocalPixelization &lpix,
             bool partial_pixelization, py::object errword, uintptr_t stream) {
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              Array<uint> e = to_array<uint>(errword, "errword");
              py::gil_scoped_release rel;
              launch_unplanned_tod2map_async(m_, t, x, lpix, partial_pixelization, e.data, (cudaStream_t) stream);
          },
          py::arg("local_map"), py::arg("tod"), py::arg("xpointing"), py::arg("local_pixelization"),
          py::arg("partial_pixelization"), py::arg("errword"), py::arg("stream") = 0);

    m.def("check_errword",
          [](py::object errword, uint ignore, uintptr_t stream) {
              Array<uint> e = to_array<uint>(errword, "errword");
              py::gil_scoped_release rel;
              check_errword(e.data, ignore, (cudaStream_t) stream);
          },
          py::arg("errword"), py::arg("ignore") = 0, py::arg("stream") = 0);

    m.def("reference_map2tod",
          [](py::object tod, py::object local_map, py::object xpointing, const LocalPixelization &lpix,
             bool partial_pixelization, bool accum) {
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              py::gil_scoped_release rel;
              reference_map2tod<float>(t, m_, x, lpix, partial_pixelization, accum);
          },
          py::arg("tod"), py::arg("local_map"), py::arg("xpointing"), py::arg("local_pixelization"),
          py::arg("partial_pixelization"), py::arg("accum"));

    m.def("reference_tod2map",
          [](py::object local_map, py::object tod, py::object xpointing, const LocalPixelization &lpix,
             bool partial_pixelization) {
              Array<float> m_ = to_array<float>(local_map, "local_map");
              Array<float> t = to_array<float>(tod, "tod");
              Array<float> x = to_array<float>(xpointing, "xpointing");
              py::gil_scoped_release rel;
              reference_tod2map<float>(m_, t, x, lpix, partial_pixelization);
          },
          py::arg("local_map"), py::arg("tod"), py::arg("xpointing"), py::arg("local_pixelization"),
          py::arg("partial_pixelization"));

    m.def("expand_dynamic_map",
          [](py::object global_ncells, py::object cell_offsets, py::object plan_mt) {
              Array<uint> g = to_array<uint>(global_ncells, "global_ncells");
              Array<long> c = to_array<long>(cell_offsets, "cell_offsets");
              Array<ulong> p = to_array<ulong>(plan_mt, "plan_mt");
              py::gil_scoped_release rel;
              return expand_dynamic_map(g, c, p);
          },
          py::arg("global_ncells"), py::arg("cell_offsets"), py::arg("plan_mt"));

    m.def("expand_dynamic_map2",
          [](py::object global_ncells, LocalPixelization &lpix, const PointingPlan &plan) {
              Array<uint> g = to_array<uint>(global_ncells, "global_ncells");
              py::gil_scoped_release rel;
              return expand_dynamic_map2(g, lpix, plan);
          },
          py::arg("global_ncells"), py::arg("local_pixelization"), py::arg("plan"));

    m.def("local_map_to_global",
          [](const LocalPixelization &lpix, py::object dst, py::object src) {
              Array<float> d = to_array<float>(dst, "dst");
              Array<float> s = to_array<float>(src, "src");
              py::gil_scoped_release rel;
              local_map_to_global<float>(lpix, d, s);
          },
          py::arg("local_pixelization"), py::arg("dst"), py::arg("src"));

    // TOD preprocessing on device arrays (gpu_mm_pybind11.cu get_border_means / deglitch and the
    // ctypes entry points extract_ranges / insert_ranges / clear_ranges / clip of gpu_mm.py:1579-1607).
    m.def("get_border_means", [](py::object out, py::object signal, py::object index_map) {
        Array<float> o = to_array<float>(out, "out"), sg = to_array<float>(signal, "signal");
        Array<int> im = to_array<int>(index_map, "index_map");
        py::gil_scoped_release rel;
        get_border_means(o, sg, im);
    }, py::arg("out"), py::arg("signal"), py::arg("index_map"));
    // deglitch(signal, bvals, cumj, index_map2) as in the reference; cumj=None computes it on the device.
    m.def("deglitch", [](py::object signal, py::object bvals, py::object cumj, py::object index_map2) {
        Array<float> sg = to_array<float>(signal, "signal"), bv = to_array<float>(bvals, "bvals"), cj;
        Array<int> im = to_array<int>(index_map2, "index_map2");
        const bool given = !cumj.is_none();
        if (given)
            cj = to_array<float>(cumj, "cumj");
        py::gil_scoped_release rel;
        if (given)
            deglitch(sg, bv, cj, im);
        else
            deglitch(sg, bv, im);
    }, py::arg("signal"), py::arg("bvals"), py::arg("cumj"), py::arg("index_map2"));
    m.def("_ranges", [](int mode, py::object tod, py::object rdata, py::object ostart, py::object det,
                        py::object istart, py::object len) {
        Array<float> t = to_array<float>(tod, "tod"), r;
        Array<int> o, d = to_array<int>(det, "dets"), s0 = to_array<int>(istart, "starts"), n = to_array<int>(len, "lens");
        if (mode != 2) {
            r = to_array<float>(rdata, "junk");
            o = to_array<int>(ostart, "offs");
        }
        py::gil_scoped_release rel;
        tod_ranges(mode, t, r, o, d, s0, n);
    });
    m.def("clip", [](py::object arr, float vmin, float vmax) {
        Array<float> a = to_array<float>(arr, "arr");
        py::gil_scoped_release rel;
        clip(a, vmin, vmax);
    }, py::arg("arr"), py::arg("vmin"), py::arg("vmax"));

    // gpu_mm_pybind11.cu:195-200 (float32 maps): host (numpy) or device (CUDA) cell-major buffers.
    m.def("cell_broadcast",
          [](py::object dst, py::object src, py::object index_map) {
              Array<float> d = to_array<float>(dst, "dst");
              Array<float> s = to_array<float>(src, "src");
              Array<long> im = to_array<long>(index_map, "index_map");
              py::gil_scoped_release rel;
              cell_broadcast<float>(d, s, im);
          },
          py::arg("dst"), py::arg("src"), py::arg("index_map"));
    m.def("cell_reduce",
          [](py::object dst, py::object src, py::object index_map) {
              Array<float> d = to_array<float>(dst, "dst");
              Array<float> s = to_array<float>(src, "src");
              Array<long> im = to_array<long>(index_map, "index_map");
              py::gil_scoped_release rel;
              cell_reduce<float>(d, s, im);
          },
          py::arg("dst"), py::arg("src"), py::arg("index_map"));
}
