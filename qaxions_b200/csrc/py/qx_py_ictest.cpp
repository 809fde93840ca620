// pyqaxions.ictest on the B200: the functions of the reference's pybind11
// module (src/examples/ictest.cxx:8-50) -- the Gaussian-soliton IC of
// src/ic/solitons.cxx:20-110 read from solitons.txt, returning Re psi[idx] --
// plus the keyword arguments dtype and path.
#include "qx_py_common.hpp"

namespace py = pybind11;
using qxpy::Box;

// 2D IC -> Re psi[idx]   (src/examples/ictest.cxx:8-25)
static double test_solitons(int N, long idx, const std::string& dtype, const std::string& path) {
    Box b(2, N, dtype, path);
    return b.psi_re(idx);
}

// 3D IC -> Re psi[idx]   (src/examples/ictest.cxx:27-42)
static double test_solitons_3D(int N, long idx, const std::string& dtype, const std::string& path) {
    Box b(3, N, dtype, path);
    return b.psi_re(idx);
}

PYBIND11_MODULE(ictest, m) {
    m.doc() = "pyqaxions.ictest (src/examples/ictest.cxx) on the B200 through the qaxions_b200 C ABI";
    m.def("test_solitons", &test_solitons, py::arg("N"), py::arg("idx"), py::arg("dtype") = "c128",
          py::arg("path") = "solitons.txt");
    m.def("test_solitons_3D", &test_solitons_3D, py::arg("N"), py::arg("idx"), py::arg("dtype") = "c128",
          py::arg("path") = "solitons.txt");
}
