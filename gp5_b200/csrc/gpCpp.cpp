// gpCpp.cpp - pybind11 module with the classes and methods of the reference's gpCpp
// (src/gpCpp.cpp:327-371), implemented as a C++ client of the C ABI in include/gp5cu.h.
//
// Differences that follow from the device-resident design:
//  * field state lives on the GPU; getTensor returns a host copy (the reference returns a
//    view of its Eigen tensor, src/pyTools.h:68-105), setTensor uploads a copy (as the
//    reference copies, src/pyTools.h:12-56);
//  * fields with the same geometry share one plan (discretisation, FFT twiddles, workspace);
//  * processorGrid / fftOrdering are accepted for signature compatibility; one GPU holds the
//    whole grid, so only [1,1,1] is meaningful;
//  * GP (gpFunctional with couplings, masses and a harmonic trap) is bound in addition to LHY
//    (the reference binds only LHY, src/gpCpp.cpp:355-358).
// Errors surface as RuntimeError, like the reference's std::runtime_error.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <array>
#include <complex>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "gp5cu.h"

namespace py = pybind11;

namespace {

void check(int st) {
    if (st != GP5_OK) throw std::runtime_error(std::string("gp5cu: ") + gp5cu_last_error());
}

using arr3d = std::array<double, 3>;
using arr3i = std::array<int, 3>;

struct PlanHandle {
    gp5cu_plan *p = nullptr;
    ~PlanHandle() {
        if (p) gp5cu_plan_destroy(p);
    }
};

// One plan per (shape, box, components, precision, device), shared by fields and models.
std::shared_ptr<PlanHandle> get_plan(const arr3i &shape, const arr3d &left, const arr3d &right, int ncomp,
                                     int precision, int device) {
    using Key = std::tuple<arr3i, arr3d, arr3d, int, int, int>;
    static std::map<Key, std::weak_ptr<PlanHandle>> cache;
    Key k{shape, left, right, ncomp, precision, device};
    auto it = cache.find(k);
    if (it != cache.end()) {
        if (auto sp = it->second.lock()) return sp;
    }
    auto h = std::make_shared<PlanHandle>();
    check(gp5cu_plan_create(&h->p, shape.data(), left.data(), right.data(), ncomp, precision, device));
    cache[k] = h;
    return h;
}

class geometry {
public:
    geometry(arr3d left, arr3d right, arr3i shape) : _left(left), _right(right), _shape(shape) {}
    const arr3d &getLeft() const { return _left; }
    const arr3d &getRight() const { return _right; }
    const arr3i &getShape() const { return _shape; }

private:
    arr3d _left, _right;
    arr3i _shape;
};

class field {
public:
    field(const geometry &geo, int nComponents, arr3i processorGrid, arr3i fftOrdering, int precision, int device)
        : _geo(geo), _nc(nComponents), _precision(precision) {
        if (processorGrid[0] * processorGrid[1] * processorGrid[2] != 1)
            throw std::runtime_error("one GPU holds the whole grid: processorGrid must be [1,1,1]");
        (void)fftOrdering;
        _plan = get_plan(geo.getShape(), geo.getLeft(), geo.getRight(), nComponents, precision, device);
        check(gp5cu_field_alloc(_plan->p, &_d));  // zero-initialised (src/gpCpp.cpp:73)
    }
    ~field() {
        if (_d) gp5cu_field_free(_plan->p, _d);
    }
    field(const field &) = delete;
    field &operator=(const field &) = delete;

    arr3i getLocalShape() const { return _geo.getShape(); }
    arr3i getOffset() const { return {0, 0, 0}; }
    int nComponents() const { return _nc; }

    py::array_t<std::complex<double>> getTensor() const {
        const auto s = _geo.getShape();
        const py::ssize_t nx = s[0], ny = s[1], nz = s[2], nc = _nc;
        const py::ssize_t e = sizeof(std::complex<double>);
        py::array_t<std::complex<double>> a({nx, ny, nz, nc}, {e, e * nx, e * nx * ny, e * nx * ny * nz});
        check(gp5cu_download_c128(_plan->p, _d, reinterpret_cast<double *>(a.mutable_data())));
        return a;
    }

    void setTensor(py::array_t<std::complex<double>, py::array::f_style | py::array::forcecast> arr) {
        const auto s = _geo.getShape();
        if (arr.ndim() != 4 || arr.shape(0) != s[0] || arr.shape(1) != s[1] || arr.shape(2) != s[2] ||
            arr.shape(3) != _nc)
            throw std::runtime_error("Unexpected rank of the python array.");
        check(gp5cu_upload_c128(_plan->p, _d, reinterpret_cast<const double *>(arr.data())));
    }

    // field::save / field::load (src/gpCpp.cpp:105-118): the reference's HDF5 layout
    // (src/io.cpp:56-256), dataset "field" [nComp][Nz][Ny][Nx] of complex (array of 2 doubles)
    void save(const std::string &filename) const {
        const auto s = _geo.getShape();
        std::vector<std::complex<double>> h((size_t)s[0] * s[1] * s[2] * _nc);
        check(gp5cu_download_c128(_plan->p, _d, reinterpret_cast<double *>(h.data())));
        const int shape[3] = {s[0], s[1], s[2]};
        check(gp5cu_h5_save_field(filename.c_str(), reinterpret_cast<const double *>(h.data()), shape, _nc));
    }
    void load(const std::string &filename) {
        const auto s = _geo.getShape();
        std::vector<std::complex<double>> h((size_t)s[0] * s[1] * s[2] * _nc);
        const int shape[3] = {s[0], s[1], s[2]};
        check(gp5cu_h5_load_field(filename.c_str(), reinterpret_cast<double *>(h.data()), shape, _nc));
        check(gp5cu_upload_c128(_plan->p, _d, reinterpret_cast<const double *>(h.data())));
    }

    double getNorm(int c) const {
        double n = 0;
        check(gp5cu_norm(_plan->p, _d, c, &n));
        return n;
    }
    void normalize(int component, double N) { check(gp5cu_normalize(_plan->p, _d, component, N)); }
    double maxDensity() const {
        double m = 0;
        check(gp5cu_max_density(_plan->p, _d, &m));
        return m;
    }

    gp5cu_plan *plan() const { return _plan->p; }
    std::shared_ptr<PlanHandle> planHandle() const { return _plan; }
    void *data() const { return _d; }
    const geometry &geo() const { return _geo; }

private:
    geometry _geo;
    int _nc;
    int _precision;
    std::shared_ptr<PlanHandle> _plan;
    void *_d = nullptr;
};

// gpCpp.cpp:289-313: labels of the droplets of component 0 with density above the cutoff
class decomposition {
public:
    py::array_t<int> decompose(const field &psi, double densityCutOff) {
        const auto s = psi.geo().getShape();
        const py::ssize_t nx = s[0], ny = s[1], nz = s[2], nc = psi.nComponents();
        const py::ssize_t e = sizeof(int);
        py::array_t<int> a({nx, ny, nz, nc}, {e, e * nx, e * nx * ny, e * nx * ny * nz});
        int k = 0;
        check(gp5cu_decompose_host(psi.plan(), psi.data(), 0, densityCutOff, a.mutable_data(), &k));
        return a;
    }
};

class model {
public:
    virtual ~model() {
        if (_f) gp5cu_functional_destroy(_f);
    }
    // functional::apply(old, new, t) (src/gpCpp.cpp:167-171)
    void apply(field &source, field &dest, double time) {
        (void)time;
        if (source.plan() != _plan->p || dest.plan() != _plan->p)
            throw std::runtime_error("fields and model belong to different geometries");
        if (&source == &dest) throw std::runtime_error("source and destination must differ");
        py::gil_scoped_release nogil;
        check(gp5cu_apply_H(_f, source.data(), dest.data()));
        check(gp5cu_plan_synchronize(_plan->p));
    }
    py::dict observables(field &psi) {
        gp5cu_observables_t o{};
        check(gp5cu_observables(_f, psi.data(), &o));
        py::dict d;
        d["norm"] = o.norm;
        d["energy"] = o.energy;
        d["ekin"] = o.ekin;
        d["epot"] = o.epot;
        d["eint"] = o.eint;
        d["mu"] = o.mu;
        d["residual"] = o.residual;
        return d;
    }
    int nComponents() const { return _nc; }
    gp5cu_functional *functional() const { return _f; }
    gp5cu_plan *plan() const { return _plan->p; }

protected:
    void init(field &psi, const gp5cu_functional_desc &d) {
        _plan = psi.planHandle();
        _nc = psi.nComponents();
        check(gp5cu_functional_create(_plan->p, &d, &_f));
    }
    std::shared_ptr<PlanHandle> _plan;
    gp5cu_functional *_f = nullptr;
    int _nc = 1;
};

// LHY droplet (src/gpCpp.cpp:178-199), with the cubic/quartic coefficients exposed
class LHY : public model {
public:
    LHY(field &psi, double c3, double c4) {
        if (psi.nComponents() != 1) throw std::runtime_error("Field should have one component");
        gp5cu_functional_desc d;
        gp5cu_functional_desc_init(&d);
        d.kind = GP5_FUNC_LHY;
        d.c3 = c3;
        d.c4 = c4;
        init(psi, d);
    }
};

// gpFunctional (src/functional.cpp:13-102): couplings g_ij, masses, harmonic trap
class GP : public model {
public:
    GP(field &psi, std::vector<std::vector<double>> couplings, std::vector<double> masses,
       std::vector<arr3d> omegas) {
        const int nc = psi.nComponents();
        gp5cu_functional_desc d;
        gp5cu_functional_desc_init(&d);
        d.kind = GP5_FUNC_GP;
        if (!couplings.empty()) {
            if ((int)couplings.size() != nc) throw std::runtime_error("Incompatible number of components");
            for (int i = 0; i < nc; i++) {
                if ((int)couplings[i].size() != nc) throw std::runtime_error("Incompatible number of components");
                for (int j = 0; j < nc; j++) d.couplings[i * 2 + j] = couplings[i][j];
            }
            d.has_couplings = 1;
        }
        for (int c = 0; c < (int)masses.size() && c < 2; c++) d.masses[c] = masses[c];
        if (!omegas.empty()) {
            if ((int)omegas.size() != nc) throw std::runtime_error("one omega triple per component");
            d.potential = GP5_POT_HARMONIC;
            for (int c = 0; c < nc; c++)
                for (int k = 0; k < 3; k++) d.omegas[c][k] = omegas[c][k];
        }
        init(psi, d);
    }
};

// timeStepper (src/gpCpp.cpp:202-287)
class timeStepper {
public:
    timeStepper(double timeStep, const std::string &stepperName, bool isImaginary)
        : _dt(timeStep), _imag(isImaginary) {
        if (stepperName == "eulero" || stepperName == "Eulero" || stepperName == "euler") _kind = GP5_STEP_EULER;
        else if (stepperName == "RK4") _kind = GP5_STEP_RK4;
        else throw std::runtime_error("Unknown stepper " + stepperName);
    }
    ~timeStepper() {
        if (_st) gp5cu_stepper_destroy(_st);
    }
    void setFunctional(model &m) {
        double t = 0;
        if (_st) {
            gp5cu_stepper_get_time(_st, &t);
            gp5cu_stepper_destroy(_st);
            _st = nullptr;
        }
        check(gp5cu_stepper_create(m.functional(), _kind, _dt, _imag ? 1 : 0, &_st));
        check(gp5cu_stepper_set_time(_st, t));
        _plan = m.plan();
        if (!_norms.empty()) check(gp5cu_stepper_set_renormalization(_st, (int)_norms.size(), _norms.data()));
        if (_compensate) check(gp5cu_stepper_set_compensation(_st, 1));
        if (_sround >= 0) check(gp5cu_stepper_set_stochastic_rounding(_st, _sround));
    }
    // extension (no reference counterpart): compensated complex64 state update, see
    // gp5cu_stepper_set_compensation; kept across setFunctional
    void setCompensation(bool on) {
        _compensate = on;
        if (_st) check(gp5cu_stepper_set_compensation(_st, on ? 1 : 0));
    }
    // extension: stochastically rounded complex64 state update (the complex64 default), see
    // gp5cu_stepper_set_stochastic_rounding; kept across setFunctional
    void setStochasticRounding(bool on) {
        _sround = on ? 1 : 0;
        if (_st) check(gp5cu_stepper_set_stochastic_rounding(_st, _sround));
    }
    void setRenormalization(const std::vector<double> &normalizations) {
        _norms = normalizations;
        if (_st) check(gp5cu_stepper_set_renormalization(_st, (int)_norms.size(), _norms.data()));
    }
    void unsetRenormalization() {
        _norms.clear();
        if (_st) check(gp5cu_stepper_set_renormalization(_st, 0, nullptr));
    }
    void advance(field &f, int nSteps) {
        if (!_st) throw std::runtime_error("setFunctional must be called before advance");
        if (f.plan() != _plan) throw std::runtime_error("field and functional belong to different geometries");
        py::gil_scoped_release nogil;
        check(gp5cu_stepper_advance(_st, f.data(), nSteps));
    }
    double getTime() const {
        double t = 0;
        if (_st) gp5cu_stepper_get_time(_st, &t);
        return t;
    }

private:
    double _dt;
    bool _imag;
    int _kind = GP5_STEP_RK4;
    gp5cu_stepper *_st = nullptr;
    gp5cu_plan *_plan = nullptr;
    std::vector<double> _norms;
    bool _compensate = false;
    int _sround = -1;  // -1: the stepper's default
};

}  // namespace

PYBIND11_MODULE(gpCpp, m) {
    m.doc() = "B200 pseudo-spectral GP stepper: the reference's gpCpp interface over the gp5cu C ABI";
    m.attr("C128") = GP5_C128;
    m.attr("C64") = GP5_C64;
    py::class_<geometry>(m, "geometry")
        .def(py::init<arr3d, arr3d, arr3i>())
        .def("getLeft", &geometry::getLeft)
        .def("getRight", &geometry::getRight)
        .def("getShape", &geometry::getShape);
    py::class_<field>(m, "field")
        .def(py::init<const geometry &, int, arr3i, arr3i, int, int>(), py::arg("geo"), py::arg("nComponents"),
             py::arg("processorGrid"), py::arg("fftOrdering"), py::arg("precision") = (int)GP5_C128,
             py::arg("device") = 0)
        .def("getLocalShape", &field::getLocalShape)
        .def("getTensor", &field::getTensor)
        .def("setTensor", &field::setTensor)
        .def("getOffset", &field::getOffset)
        .def("getNorm", &field::getNorm)
        .def("normalize", &field::normalize)
        .def("save", &field::save)
        .def("load", &field::load)
        .def("maxDensity", &field::maxDensity);
    py::class_<model>(m, "model")
        .def("apply", &model::apply)
        .def("observables", &model::observables)
        .def("nComponents", &model::nComponents);
    py::class_<LHY, model>(m, "LHY")
        .def(py::init<field &, double, double>(), py::arg("psi"), py::arg("c3") = -3.0, py::arg("c4") = 2.5);
    py::class_<GP, model>(m, "GP")
        .def(py::init<field &, std::vector<std::vector<double>>, std::vector<double>, std::vector<arr3d>>(),
             py::arg("psi"), py::arg("couplings") = std::vector<std::vector<double>>{},
             py::arg("masses") = std::vector<double>{}, py::arg("omegas") = std::vector<arr3d>{});
    py::class_<decomposition>(m, "decomposition")
        .def(py::init<>())
        .def("decompose", &decomposition::decompose, py::arg("psi"), py::arg("densityCutOff"));
    py::class_<timeStepper>(m, "timeStepper")
        .def(py::init<double, std::string, bool>())
        .def("setRenormalization", &timeStepper::setRenormalization)
        .def("setCompensation", &timeStepper::setCompensation)
        .def("setStochasticRounding", &timeStepper::setStochasticRounding)
        .def("unsetRenormalization", &timeStepper::unsetRenormalization)
        .def("setFunctional", &timeStepper::setFunctional)
        .def("advance", &timeStepper::advance)
        .def("getTime", &timeStepper::getTime);
}
