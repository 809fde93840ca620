// pyqaxions.fieldtest on the B200: the functions of the reference's pybind11
// module (src/examples/fieldtest.cxx:11-105) with the same names, positional
// arguments and return values, plus the keyword arguments dtype ("c128" FP64,
// "c64" fused FP32) and path (the soliton file).
#include "qx_py_common.hpp"

namespace py = pybind11;
using qxpy::Box;

// updatePotential; kick(dt) -> Re psi[idx]   (src/examples/fieldtest.cxx:11-30)
static double test_kick(int n, int N, double dt, long idx, const std::string& dtype, const std::string& path) {
    Box b(n, N, dtype, path);
    b.call(qx_update_potential(b.h()));
    b.call(qx_kick(b.h(), dt));
    return b.psi_re(idx);
}

// drift(dt) -> Re psi[idx]   (src/examples/fieldtest.cxx:32-50)
static double test_drift(int n, int N, double dt, long idx, const std::string& dtype, const std::string& path) {
    Box b(n, N, dtype, path);
    b.call(qx_drift(b.h(), dt));
    return b.psi_re(idx);
}

// updatePotential -> V[idx]   (src/examples/fieldtest.cxx:53-71)
static double test_potential(int n, int N, long idx, const std::string& dtype, const std::string& path) {
    Box b(n, N, dtype, path);
    b.call(qx_update_potential(b.h()));
    return b.V(idx);
}

// updatePotential; kick(dt/2); drift(dt); updatePotential; kick(dt/2)
// -> Re psi[idx]   (src/examples/fieldtest.cxx:73-96)
static double test_kick_drift_step(int n, int N, double dt, long idx, const std::string& dtype,
                                   const std::string& path) {
    Box b(n, N, dtype, path);
    b.call(qx_update_potential(b.h()));
    b.call(qx_kick(b.h(), 0.5 * dt));
    b.call(qx_drift(b.h(), dt));
    b.call(qx_update_potential(b.h()));
    b.call(qx_kick(b.h(), 0.5 * dt));
    return b.psi_re(idx);
}

PYBIND11_MODULE(fieldtest, m) {
    m.doc() = "pyqaxions.fieldtest (src/examples/fieldtest.cxx) on the B200 through the qaxions_b200 C ABI";
    m.def("test_kick", &test_kick, py::arg("n"), py::arg("N"), py::arg("dt"), py::arg("idx"),
          py::arg("dtype") = "c128", py::arg("path") = "solitons.txt");
    m.def("test_drift", &test_drift, py::arg("n"), py::arg("N"), py::arg("dt"), py::arg("idx"),
          py::arg("dtype") = "c128", py::arg("path") = "solitons.txt");
    m.def("test_potential", &test_potential, py::arg("n"), py::arg("N"), py::arg("idx"),
          py::arg("dtype") = "c128", py::arg("path") = "solitons.txt");
    m.def("test_kick_drift_step", &test_kick_drift_step, py::arg("n"), py::arg("N"), py::arg("dt"), py::arg("idx"),
          py::arg("dtype") = "c128", py::arg("path") = "solitons.txt");
}
