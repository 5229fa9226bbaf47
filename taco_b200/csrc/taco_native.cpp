// taco_native.cpp -- pybind11 module `_taco_native`: the reference's Python module name
// (cpp/python/_taco_native.cpp:6-9 exposes version()), here wrapping the C-ABI of
// libtaco_b200.so for host (numpy) buffers.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "taco_b200.h"

namespace py = pybind11;
using c128 = std::complex<double>;

namespace {

void check(int rc) {
    if (rc == TACO_OK) return;
    const std::string msg = taco_last_error();
    if (rc == TACO_ERR_INVALID_ARGUMENT) throw py::value_error(msg);
    if (rc == TACO_ERR_OUT_OF_RANGE) throw py::index_error(msg);
    throw std::runtime_error("[" + std::to_string(rc) + "] " + msg);
}

struct View {
    py::array_t<double, py::array::c_style | py::array::forcecast> omegas;
    py::array_t<int32_t, py::array::c_style | py::array::forcecast> mirror, p2f;
    py::array_t<c128, py::array::c_style | py::array::forcecast> ops;
    taco_system_view v{};
};

// pair_to_freq and ops are given column-major (as the C-ABI); ops: [num_ops, N*N].
View make_view(int N, py::array omegas, py::object mirror, py::array p2f_colmajor, py::array ops_colmajor, double tol) {
    View w;
    w.omegas = omegas;
    w.p2f = p2f_colmajor;
    w.ops = ops_colmajor;
    w.v.N = N;
    w.v.nf = static_cast<int>(w.omegas.size());
    w.v.num_ops = N > 0 ? static_cast<int>(w.ops.size() / (static_cast<size_t>(N) * N)) : 0;
    w.v.omegas = w.omegas.data();
    w.v.pair_to_freq = w.p2f.data();
    w.v.ops = reinterpret_cast<const taco_c128*>(w.ops.data());
    w.v.tol = tol;
    if (!mirror.is_none()) {
        w.mirror = mirror;
        w.v.mirror = w.mirror.data();
    }
    return w;
}

}  // namespace

PYBIND11_MODULE(_taco_native, m) {
    m.doc() = "pybind11 wrapper of the taco_b200 C-ABI (host buffers)";
    m.def("version", [] { return std::string(taco_version()); });
    m.def("set_fcr_fft_pad_factor", [](size_t f) { taco_set_fcr_fft_pad_factor(f); });
    m.def("get_fcr_fft_pad_factor", [] { return taco_get_fcr_fft_pad_factor(); });
    m.def(
        "build_tcl4_generator_batch",
        [](int N, py::array omegas, py::object mirror, py::array p2f, py::array ops, double tol,
           py::array_t<c128, py::array::c_style | py::array::forcecast> gamma, double dt,
           py::array_t<uint32_t, py::array::c_style | py::array::forcecast> tidx, int precision) -> py::tuple {
            View w = make_view(N, omegas, mirror, p2f, ops, tol);
            const size_t Nt = gamma.ndim() == 2 ? static_cast<size_t>(gamma.shape(1)) : 0;
            const size_t T = tidx.size() ? static_cast<size_t>(tidx.size()) : Nt;
            const size_t E = static_cast<size_t>(N) * N * N * N;
            double fcr_ms = 0.0;
            if (precision == TACO_PREC_FP64) {
                py::array_t<c128> out({T, E});
                check(taco_tcl4_build_batch(&w.v, reinterpret_cast<const taco_c128*>(gamma.data()), Nt, dt,
                                            tidx.size() ? tidx.data() : nullptr, tidx.size(), TACO_FCR_CONVOLUTION,
                                            precision, out.mutable_data(), 0, nullptr, &fcr_ms));
                return py::tuple(py::make_tuple(out, fcr_ms));
            }
            py::array_t<std::complex<float>> out({T, E});
            check(taco_tcl4_build_batch(&w.v, reinterpret_cast<const taco_c128*>(gamma.data()), Nt, dt,
                                        tidx.size() ? tidx.data() : nullptr, tidx.size(), TACO_FCR_CONVOLUTION,
                                        precision, out.mutable_data(), 0, nullptr, &fcr_ms));
            return py::tuple(py::make_tuple(out, fcr_ms));
        },
        "L4 at the requested times: ([T, N^4] column-major matrices, fcr_ms)");
    m.def(
        "compute_triple_kernels",
        [](int N, py::array omegas, py::object mirror, py::array p2f, double tol,
           py::array_t<c128, py::array::c_style | py::array::forcecast> gamma, double dt) {
            py::array_t<c128> none_ops(0);
            View w = make_view(N, omegas, mirror, p2f, none_ops, tol);
            const size_t nf = static_cast<size_t>(gamma.shape(0)), Nt = static_cast<size_t>(gamma.shape(1));
            std::vector<size_t> shape{nf * nf * nf, Nt};
            py::array_t<c128> F(shape), C(shape), R(shape);
            check(taco_compute_triple_kernels(&w.v, reinterpret_cast<const taco_c128*>(gamma.data()), Nt, dt,
                                              TACO_FCR_CONVOLUTION, reinterpret_cast<taco_c128*>(F.mutable_data()),
                                              reinterpret_cast<taco_c128*>(C.mutable_data()),
                                              reinterpret_cast<taco_c128*>(R.mutable_data()), 0, nullptr));
            return py::make_tuple(F, C, R);
        });
    m.def(
        "rk4_propagate",
        [](py::array_t<c128, py::array::c_style | py::array::forcecast> L_colmajor,
           py::array_t<c128, py::array::c_style | py::array::forcecast> r0, double dt) {
            const size_t steps = static_cast<size_t>(L_colmajor.shape(0)) - 1;
            const int D = static_cast<int>(L_colmajor.shape(1));
            py::array_t<c128> r(static_cast<size_t>(D));
            std::copy(r0.data(), r0.data() + D, r.mutable_data());
            check(taco_rk4_propagate(L_colmajor.data(), nullptr, nullptr, 0, steps, D, dt,
                                     reinterpret_cast<taco_c128*>(r.mutable_data()), 0, nullptr, nullptr, nullptr, 0,
                                     nullptr));
            return r;
        },
        "RK4 over [steps+1, D, D] column-major generators (L[k].T in numpy terms)");
}
