// py_ctomocam.cpp -- pybind11 module `cTomocam` with the reference binding's
// names and signatures (src/pyTomocam.cpp:81-152), implemented on the C ABI
// of include/tomocam_b200.h.
//
// Like the reference: float32 C-contiguous arrays (np_array_t is c_style,
// src/pyTomocam.cpp:38), 2-D input treated as one slice (:53-68), 3-D
// output, failures raise RuntimeError.  Unlike the reference the GIL is
// released around device work and no output buffer leaks.
//
// The reference's Python layer (tomocam/transform.py, modeling.py,
// gradients.py) calls radon_adj, gradients and total_variation, which its
// binding never defined; they are provided here with the meaning those
// Python functions document.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "tomocam_b200.h"

namespace py = pybind11;
using farr = py::array_t<float, py::array::c_style | py::array::forcecast>;
using darr = py::array_t<double, py::array::c_style | py::array::forcecast>;

static void check(int rc) {
    if (rc != TC_OK) throw std::runtime_error(tc_last_error_string());
}

struct Dims {
    int s, r, c;
};

static Dims dims3(const farr &a, const char *what) {
    if (a.ndim() == 2) return {1, (int)a.shape(0), (int)a.shape(1)};
    if (a.ndim() == 3) return {(int)a.shape(0), (int)a.shape(1), (int)a.shape(2)};
    throw std::runtime_error(std::string(what) + " must be a 2-D or 3-D array");
}

static std::vector<float> angles_of(const farr &a) {
    return std::vector<float>(a.data(), a.data() + a.size());
}

// device buffer RAII for the binding-level helpers
struct Dev {
    float *p = nullptr;
    explicit Dev(size_t n) {
        if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error("device allocation failed");
        }
    }
    ~Dev() {
        if (p) cudaFree(p);
    }
    void up(const float *h, size_t n) {
        if (cudaMemcpy(p, h, n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("host to device copy failed");
    }
    void down(float *h, size_t n) const {
        if (cudaMemcpy(h, p, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("device to host copy failed");
    }
};

struct Plan {
    tc_plan *p = nullptr;
    Plan(int n, const std::vector<float> &ang, int flags) {
        tc_geom g{n, (int)ang.size(), ang.data(), 0.0, 0, flags};
        check(tc_plan_create(&g, &p));
    }
    ~Plan() { tc_plan_destroy(p); }
};

// cTomocam.radon(imgstack, angs) -> [S, P, N]   (src/pyTomocam.cpp:81-92)
// center / over_sample are accepted for tomocam/transform.py:4-26, which
// passes them; the reference's forward projection has no centre shift.
static farr radon(const farr &img, const farr &angs, py::object center, py::object over_sample) {
    (void)center;
    (void)over_sample;
    Dims d = dims3(img, "imgstack");
    if (d.r != d.c) throw std::runtime_error("images must be square");
    auto ang = angles_of(angs);
    farr out({(py::ssize_t)d.s, (py::ssize_t)ang.size(), (py::ssize_t)d.c});
    const float *ip = img.data();
    float *op = out.mutable_data();
    int rc;
    {
        py::gil_scoped_release nogil;
        rc = tc_radon_host(ip, d.s, d.c, ang.data(), (int)ang.size(), op);
    }
    check(rc);
    return out;
}

// cTomocam.backproject(sino, angs, cen) -> [S, D, D]   (src/pyTomocam.cpp:94-114)
static farr backproject(const farr &sino, const farr &angs, float cen) {
    Dims d = dims3(sino, "sino");
    auto ang = angles_of(angs);
    if ((int)ang.size() != d.r) throw std::runtime_error("number of angles does not match sinogram");
    farr out({(py::ssize_t)d.s, (py::ssize_t)d.c, (py::ssize_t)d.c});
    const float *ip = sino.data();
    float *op = out.mutable_data();
    int rc;
    {
        py::gil_scoped_release nogil;
        rc = tc_backproject_host(ip, d.s, d.r, d.c, ang.data(), cen, op);
    }
    check(rc);
    return out;
}

// cTomocam.radon_adj(sino, angs, center, over_sample): the back-projection
// tomocam/transform.py:29-53 documents (over_sample accepted, the fine grid is 2x)
static farr radon_adj(const farr &sino, const farr &angs, float center, py::object over_sample) {
    (void)over_sample;
    return backproject(sino, angs, center);
}

// cTomocam.mbir(sino, angles, center, num_iters, sigma, tol, xtol)  (src/pyTomocam.cpp:116-134)
static farr mbir(const farr &sino, const farr &angs, float center, int num_iters, float sigma,
                 float tol, float xtol, float p, float prior_weight, int use_graph, int verbose) {
    Dims d = dims3(sino, "sino");
    auto ang = angles_of(angs);
    if ((int)ang.size() != d.r) throw std::runtime_error("number of angles does not match sinogram");
    farr out({(py::ssize_t)d.s, (py::ssize_t)d.c, (py::ssize_t)d.c});
    tc_mbir_opts o;
    tc_mbir_opts_default(&o);
    o.p = p;
    o.prior_weight = prior_weight;
    o.use_graph = use_graph;
    o.verbose = verbose;
    const float *ip = sino.data();
    float *op = out.mutable_data();
    int rc;
    {
        py::gil_scoped_release nogil;
        rc = tc_mbir_host(ip, d.s, d.r, d.c, ang.data(), center, num_iters, sigma, tol, xtol, op, &o);
    }
    check(rc);
    return out;
}

// cTomocam.gradients(model, sinogram, angles, center, over_sample): the data
// gradient A^T (A x - y) that tomocam/modeling.py:5-24 documents, computed
// with the NUFFT operators on the model's grid.
static farr gradients(const farr &model, const farr &sino, const farr &angs, float center,
                      py::object over_sample) {
    (void)center;
    (void)over_sample;
    Dims dm = dims3(model, "model"), ds = dims3(sino, "sinogram");
    auto ang = angles_of(angs);
    if (dm.r != dm.c || ds.s != dm.s || ds.c != dm.c || ds.r != (int)ang.size())
        throw std::runtime_error("model / sinogram / angles shapes do not match");
    const size_t nx = (size_t)dm.s * dm.c * dm.c, ny = (size_t)ds.s * ds.r * ds.c;
    farr out({(py::ssize_t)dm.s, (py::ssize_t)dm.c, (py::ssize_t)dm.c});
    std::vector<float> hx(model.data(), model.data() + nx), hy(sino.data(), sino.data() + ny);
    float *op = out.mutable_data();
    {
        py::gil_scoped_release nogil;
        Plan pl(dm.c, ang, TC_PLAN_NO_PSF);
        Dev dx(nx), dy(ny), dr(ny);
        dx.up(hx.data(), nx);
        dy.up(hy.data(), ny);
        check(tc_radon(pl.p, dx.p, dr.p, dm.s, nullptr));
        check(tc_axpby(-1.0f, dy.p, 1.0f, dr.p, ny, nullptr));  // r = A x - y
        check(tc_iradon(pl.p, dr.p, dx.p, dm.s, 0, nullptr));
        dx.down(op, nx);
    }
    return out;
}

// cTomocam.toeplitz_gradients(model, sinoT, psf): H x - A^T y with a given
// point-spread function (tomocam/gradients.py:5-28)
static farr toeplitz_gradients(const farr &model, const farr &sinoT, const darr &psf) {
    Dims dm = dims3(model, "model"), dt = dims3(sinoT, "sinoT");
    if (dm.r != dm.c || dt.s != dm.s || dt.r != dm.r || dt.c != dm.c)
        throw std::runtime_error("model and sinoT shapes do not match");
    const int n = dm.c;
    if (psf.ndim() != 2 || psf.shape(0) != 2 * n - 1 || psf.shape(1) != 2 * n - 1)
        throw std::runtime_error("psf must be (2N-1, 2N-1)");
    const size_t nx = (size_t)dm.s * n * n;
    farr out({(py::ssize_t)dm.s, (py::ssize_t)n, (py::ssize_t)n});
    const float *mp = model.data();
    const float *tp = sinoT.data();
    const double *pp = psf.data();
    float *op = out.mutable_data();
    {
        py::gil_scoped_release nogil;
        std::vector<float> one_angle(1, 0.0f);
        Plan pl(n, one_angle, TC_PLAN_NO_PSF);
        check(tc_plan_set_psf(pl.p, pp));
        Dev dx(nx), dt2(nx), dg(nx);
        dx.up(mp, nx);
        dt2.up(tp, nx);
        check(tc_toeplitz_grad(pl.p, dx.p, dt2.p, dg.p, dm.s, nullptr, nullptr, nullptr));
        dg.down(op, nx);
    }
    return out;
}

// cTomocam.total_variation(gradients, model, sigma, p=1.2): in-place
// g += qGGMRF'(model) (add_total_var2, src/tv_update.cpp:76-106)
static void total_variation(farr &grad, const farr &model, float sigma, float p) {
    Dims dg = dims3(grad, "gradients"), dm = dims3(model, "model");
    if (dg.s != dm.s || dg.r != dm.r || dg.c != dm.c)
        throw std::runtime_error("gradients and model shapes do not match");
    const size_t n = (size_t)dm.s * dm.r * dm.c;
    float *gp = grad.mutable_data();
    const float *mp = model.data();
    {
        py::gil_scoped_release nogil;
        Dev dx(n), dgr(n);
        dx.up(mp, n);
        dgr.up(gp, n);
        check(tc_qggmrf_grad(dx.p, dgr.p, dm.s, dm.r, dm.c, sigma, p, 1.0f, nullptr));
        dgr.down(gp, n);
    }
}

PYBIND11_MODULE(cTomocam, m) {
    m.doc() = "tomocam-b200: B200 implementation of tomoCAM's MBIR path";
    m.def("set_num_of_gpus", [](int n) { check(tc_set_num_of_gpus(n)); }, py::arg("num"));
    m.def("radon", &radon, py::arg("imgstack"), py::arg("angs"), py::arg("center") = py::none(),
          py::arg("over_sample") = py::none());
    m.def("backproject", &backproject, py::arg("sino"), py::arg("angs"), py::arg("cen"));
    m.def("radon_adj", &radon_adj, py::arg("sino"), py::arg("angs"), py::arg("center"),
          py::arg("over_sample") = py::none());
    m.def("mbir", &mbir, "Model-based iterative reconstruction", py::arg("sino"),
          py::arg("angles"), py::arg("center"), py::arg("num_iters"), py::arg("sigma"),
          py::arg("tol"), py::arg("xtol"), py::arg("p") = 1.2f, py::arg("prior_weight") = 1.0f,
          py::arg("use_graph") = 1, py::arg("verbose") = 0);
    m.def("gradients", &gradients, py::arg("model"), py::arg("sinogram"), py::arg("angles"),
          py::arg("center") = 0.0f, py::arg("over_sample") = py::none());
    m.def("toeplitz_gradients", &toeplitz_gradients, py::arg("model"), py::arg("sinoT"),
          py::arg("psf"));
    m.def("total_variation", &total_variation, py::arg("gradients"), py::arg("model"),
          py::arg("sigma"), py::arg("p") = 1.2f);
    m.def("version", []() { return std::string(tc_version()); });
}
