// qx_py_common.hpp -- shared part of the pybind11 test modules
// pyqaxions.fieldtest / pyqaxions.ictest (qx_py_fieldtest.cpp,
// qx_py_ictest.cpp).  They call the library only through its C ABI
// (include/qaxions_b200.h), as any other binding would.
//
// Every function builds a box the way the reference's examples do
// (src/examples/fieldtest.cxx:11-23): defaults() (src/parse.cxx:7-29) with N,
// dim and norm = 1, so pref = 4 pi norm a = 4 pi (src/field.cxx:78,298),
// rho_mean = 1, L = 1; the Gaussian-soliton IC read from `path`
// (solitons.txt in the working directory, src/ic/solitons.cxx:32) over the
// background sol_bkg = 1 (src/parse.cxx:20).  dtype "c128" is the plain FP64
// form, "c64" the fused FP32 form.
#pragma once

#include <pybind11/pybind11.h>

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/qaxions_b200.h"

namespace qxpy {

namespace py = pybind11;

// owns one qx_field_t; a non-zero status becomes a Python exception
class Box {
  public:
    Box(int dim, int N, const std::string& dtype, const std::string& path) {
        int dt;
        if (dtype == "c128") dt = QX_C128;
        else if (dtype == "c64") dt = QX_C64;
        else throw py::value_error("dtype must be 'c128' or 'c64'");
        const double pref = 4.0 * M_PI * 1.0;  // 4 pi norm, norm = 1
        check(qx_create(dim, N, 1.0, pref, 1.0, dt, QX_K0_REFERENCE, 1e-4, &h_), nullptr);
        check(qx_ic_solitons_file(h_, path.c_str(), 1.0), h_);
        dim_ = dim;
        N_ = N;
    }
    ~Box() {
        if (h_) qx_destroy(h_);
    }
    Box(const Box&) = delete;
    Box& operator=(const Box&) = delete;

    qx_field_t* h() const { return h_; }

    // Field::getPsiIdx (src/field.h:37): Re psi at flat index idx
    double psi_re(long idx) {
        std::vector<double> p(2 * sites());
        check(qx_get_psi(h_, p.data()), h_);
        return p.at(2 * (size_t)index(idx));
    }
    // Field::getVIdx (src/field.h:42)
    double V(long idx) {
        std::vector<double> v(sites());
        check(qx_get_V(h_, v.data()), h_);
        return v.at((size_t)index(idx));
    }
    void call(int status) { check(status, h_); }

  private:
    size_t sites() const { return (size_t)std::pow((double)N_, dim_); }
    long index(long idx) const {
        if (idx < 0 || (size_t)idx >= sites()) throw py::index_error("idx out of range");
        return idx;
    }
    static void check(int status, qx_field_t* h) {
        if (status == QX_OK) return;
        const std::string msg = qx_last_error(h) ? qx_last_error(h) : "";
        if (status == QX_ERR_INVALID) throw py::value_error(msg);
        if (status == QX_ERR_NOMEM) throw std::bad_alloc();
        throw std::runtime_error("[qx status " + std::to_string(status) + "] " + msg);
    }

    qx_field_t* h_ = nullptr;
    int dim_ = 0, N_ = 0;
};

}  // namespace qxpy
