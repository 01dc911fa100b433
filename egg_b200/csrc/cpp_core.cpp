// pybind11 module `cpp_core`: the reference's Python-facing surface
// (src/bindings.cpp:1541-2130, module egg._cpp.cpp_core) over the egg_b200
// C-ABI.  Dict/array unpacking and argument checks live here; every numeric
// operation runs on the GPU through libegg_b200.so.  Python passes float64 and
// gets float64 back, as in the reference.
#include "egg_b200.h"

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace py = pybind11;

namespace
{

using IArr = py::array_t<int32_t, py::array::c_style | py::array::forcecast>;
using DArr = py::array_t<double, py::array::c_style | py::array::forcecast>;

[[noreturn]] void raise_status(int st)
{
    const std::string msg = egg_b200_last_error();
    if (st == EGG_B200_EINVAL) { throw py::value_error(msg); }
    if (st == EGG_B200_ENOTSUP) {
        PyErr_SetString(PyExc_NotImplementedError, msg.c_str());
        throw py::error_already_set();
    }
    throw std::runtime_error(msg);
}

void check(int st)
{
    if (st != EGG_B200_OK) { raise_status(st); }
}

// Default arithmetic of sessions created without `precision=` (every session
// a reference caller creates): EGG_B200_PRECISION=mixed selects fp32 bulk;
// anything else (or unset) is plain fp64, the reference's double build.  Read
// once, at the first use (module import), so that REAL_IS_FLOAT -- the
// reference's "this core computes in float" -- holds for every such session.
int default_precision()
{
    static const int prec = [] {
        const char* v = std::getenv("EGG_B200_PRECISION");
        if (v && (std::string(v) == "mixed" || std::string(v) == "fp32")) { return int(EGG_B200_PREC_MIXED); }
        return int(EGG_B200_PREC_FP64);
    }();
    return prec;
}

int parse_precision(const py::object& p)
{
    if (p.is_none()) { return default_precision(); }
    const std::string s = p.cast<std::string>();
    if (s == "fp64" || s == "double") { return EGG_B200_PREC_FP64; }
    if (s == "mixed" || s == "fp32") { return EGG_B200_PREC_MIXED; }
    throw py::value_error("precision must be 'fp64' or 'mixed', got '" + s + "'");
}

int objective_of(const std::string& phase)
{
    if (phase == "untangle") { return EGG_B200_OBJ_UNTANGLE; }
    if (phase == "shape_size") { return EGG_B200_OBJ_SHAPE_SIZE; }
    return EGG_B200_OBJ_SHAPE;
}

int device_of(const std::string& device)
{
    if (device == "cpu") {
        throw std::runtime_error(
          "select_queue: egg_b200 runs on the GPU only; device='cpu' has no implementation here "
          "(use device='gpu' or 'auto')");
    }
    if (device == "gpu" || device == "auto") { return -1; }
    if (device.rfind("cuda:", 0) == 0) { return std::stoi(device.substr(5)); }
    throw py::value_error("device must be 'auto', 'gpu' or 'cuda:N', got '" + device + "'");
}

// Keeps every numpy buffer handed to the C-ABI alive until the call returns.
struct Keep {
    std::vector<py::object> objs;
    const int32_t* ints(const py::handle& h, int64_t* n = nullptr)
    {
        IArr a = IArr::ensure(h);
        if (!a) { throw py::value_error("expected an integer array"); }
        objs.push_back(a);
        if (n) { *n = int64_t(a.size()); }
        return a.size() ? a.data() : nullptr;
    }
    const double* reals(const py::handle& h, int64_t* n = nullptr)
    {
        DArr a = DArr::ensure(h);
        if (!a) { throw py::value_error("expected a float array"); }
        objs.push_back(a);
        if (n) { *n = int64_t(a.size()); }
        return a.size() ? a.data() : nullptr;
    }
};

int64_t checked_num_nodes(const DArr& X, int d)
{
    auto buf = X.request();
    if (buf.ndim != 1) {
        throw py::value_error("X must be a flat 1-D array of length d*N; got ndim=" + std::to_string(buf.ndim) +
                              " (did you pass an (N, d) array? ravel() it first).");
    }
    if (buf.shape[0] % d != 0) {
        throw py::value_error("X length must be a multiple of d (" + std::to_string(d) +
                              " coordinates per node); got " + std::to_string(buf.shape[0]) + ".");
    }
    return int64_t(buf.shape[0]) / d;
}

// Write one byte per page of every span, on up to 16 threads (spans of
// 64 MiB or more are split), so later writes into them do not fault.
void prefault(const std::vector<std::pair<char*, size_t>>& spans)
{
    constexpr size_t kChunk = size_t(64) << 20, kPage = 4096;
    std::vector<std::pair<char*, size_t>> work;
    size_t total = 0;
    for (const auto& sp : spans) {
        for (size_t a = 0; a < sp.second; a += kChunk) { work.emplace_back(sp.first + a, std::min(kChunk, sp.second - a)); }
        total += sp.second;
    }
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t T = std::min({hw, size_t(16), std::max<size_t>(1, total >> 26)});
    auto body = [&](size_t t) {
        for (size_t i = t; i < work.size(); i += T) {
            volatile char* p = work[i].first;
            for (size_t o = 0; o < work[i].second; o += kPage) { p[o] = 0; }
        }
    };
    std::vector<std::thread> th;
    for (size_t t = 1; t < T; ++t) { th.emplace_back(body, t); }
    body(0);
    for (auto& x : th) { x.join(); }
}

struct PinnedBuf {
    void* p;
    int64_t bytes;
};

struct Desc {
    egg_b200_session_desc d {};
    Keep keep;
    std::vector<int32_t> shapes, bgd, tags;
    std::vector<double> eparams, arena;
};

// Fill the C-ABI descriptor from the reference's two dicts + X
// (src/bindings.cpp:332-489 unpack_context, :757 apply_structured_remap).
void fill_desc(Desc& D, const py::dict& ctx, const py::dict& st, const DArr& X, int dim, int prec, int dev)
{
    if (dim != 2 && dim != 3) {
        throw py::value_error("egg C++ core: dimension must be 2 or 3, got " + std::to_string(dim));
    }
    auto& d = D.d;
    d.dim = dim;
    d.precision = prec;
    d.device = dev;
    d.num_nodes = checked_num_nodes(X, dim);
    D.keep.objs.push_back(X);
    d.X = X.size() ? X.data() : nullptr;

    // structured
    py::list shapes = st["interior_shapes"].cast<py::list>();
    py::list bgd = st["block_global_dof"].cast<py::list>();
    if (py::len(bgd) != py::len(shapes)) {
        throw py::value_error("structured: block_global_dof count != interior_shapes count");
    }
    d.num_blocks = int32_t(py::len(shapes));
    for (size_t b = 0; b < py::len(shapes); ++b) {
        IArr s = IArr::ensure(shapes[b]);
        if (!s || s.size() != dim) { throw py::value_error("structured: each interior shape must have D entries"); }
        int64_t n = 1;
        for (int k = 0; k < dim; ++k) {
            D.shapes.push_back(s.data()[k]);
            n *= s.data()[k];
        }
        IArr ids = IArr::ensure(bgd[b]);
        if (!ids || int64_t(ids.size()) != n) {
            throw py::value_error("structured: block_global_dof length != prod(shape)");
        }
        D.bgd.insert(D.bgd.end(), ids.data(), ids.data() + ids.size());
    }
    d.interior_shapes = D.shapes.data();
    d.block_global_dof = D.bgd.data();
    int64_t n1 = 0, n2 = 0, n3 = 0, n4 = 0;
    d.halo_src_block = D.keep.ints(st["halo_src_block"], &n1);
    d.halo_src_padded = D.keep.ints(st["halo_src_padded"], &n2);
    d.halo_dst_block = D.keep.ints(st["halo_dst_block"], &n3);
    d.halo_dst_padded = D.keep.ints(st["halo_dst_padded"], &n4);
    if (n3 != n1 || n2 != n1 * dim || n4 != n1 * dim) { throw py::value_error("structured: halo table lengths disagree"); }
    d.num_halo = n1;
    d.sing_block = D.keep.ints(st["sing_block"], &n1);
    d.sing_logical = D.keep.ints(st["sing_logical"], &n2);
    if (n2 != n1 * dim) { throw py::value_error("structured: sing table lengths disagree"); }
    d.num_sing = n1;

    // groups: the reference merges all groups into one view; this core takes
    // exactly one group (build_flat_context emits one).
    py::list groups = ctx["groups"].cast<py::list>();
    if (py::len(groups) > 1) { throw py::value_error("unpack_context: this core takes a single DOF group"); }
    if (py::len(groups) == 1) {
        py::dict g = groups[0].cast<py::dict>();
        d.ndof = g["D"].cast<int64_t>();
        int64_t n = 0;
        d.dof_idx = D.keep.ints(g["dof_idx"], &n);
        if (n != d.ndof) { throw py::value_error("validate_context: group[0] dof_idx size " + std::to_string(n) + " != " + std::to_string(d.ndof)); }
        d.P_of = D.keep.ints(g["P_of"], &n);
        if (n != d.ndof) { throw py::value_error("validate_context: group[0] P_of size " + std::to_string(n) + " != " + std::to_string(d.ndof)); }
        if (g.contains("interior_block")) {
            d.interior_block = D.keep.ints(g["interior_block"], &n);
            if (n != d.ndof) { throw py::value_error("validate_context: group[0] interior_block size mismatch"); }
            d.interior_logical = D.keep.ints(g["interior_logical"], &n);
            if (n != d.ndof * dim) { throw py::value_error("validate_context: group[0] interior_logical size mismatch"); }
        }
        d.gc = D.keep.ints(g["gc"], &d.total_samples);
        for (int k = 0; k < dim; ++k) {
            d.gn[k] = D.keep.ints(g[("gn" + std::to_string(k)).c_str()], &n);
            if (n != d.total_samples) { throw py::value_error("validate_context: group[0] gn" + std::to_string(k) + " size mismatch"); }
            d.s[k] = D.keep.reals(g[("s" + std::to_string(k)).c_str()], &n);
            if (n != d.total_samples) { throw py::value_error("validate_context: group[0] s" + std::to_string(k) + " size mismatch"); }
        }
        d.role = D.keep.ints(g["role"], &n);
        if (n != d.total_samples) { throw py::value_error("validate_context: group[0] role size mismatch"); }
        d.W_inv = D.keep.reals(g["W_inv"], &d.W_inv_len);
        if (g.contains("weight")) { d.weight = D.keep.reals(g["weight"], &d.weight_len); }
        // Entity partitions: every DOF must be covered exactly once; non-Free
        // tags mark constrained boundary DOFs.
        D.tags.assign(size_t(d.ndof), -1);
        bool constrained = false;
        if (g.contains("entities")) {
            for (auto item : g["entities"].cast<py::dict>()) {
                py::dict ed = item.second.cast<py::dict>();
                if (!ed.contains("tag")) {
                    throw py::value_error("unpack_context: entities carries a '__blob__' group (unsupported)");
                }
                const int tag = ed["tag"].cast<int>();
                const int kf = ed.contains("kFields") ? ed["kFields"].cast<int>() : 0;
                IArr dl = IArr::ensure(ed["dof_local"]);
                DArr rec = ed.contains("records") ? DArr::ensure(ed["records"]) : DArr();
                if (tag != 0 && rec.size() != dl.size() * py::ssize_t(kf)) {
                    throw py::value_error("validate_context: entity records size " + std::to_string(rec.size()) +
                                          " != count*kFields " + std::to_string(dl.size() * kf));
                }
                // Segmented fields ({data, off} CSR per field: B-spline knots,
                // control points, weights) go to the entity arena; a B-spline
                // record then addresses its slices by arena offset.
                std::vector<int64_t> seg_base;
                std::vector<IArr> seg_off;
                if (ed.contains("seg")) {
                    for (auto sv : ed["seg"].cast<py::list>()) {
                        py::dict sd = sv.cast<py::dict>();
                        DArr data = DArr::ensure(sd["data"]);
                        IArr off = IArr::ensure(sd["off"]);
                        if (off.size() != dl.size() + 1) {
                            throw py::value_error("validate_context: entity seg off size != count + 1");
                        }
                        for (py::ssize_t r = 0; r + 1 < off.size(); ++r) {
                            if (off.data()[r] < 0 || off.data()[r] > off.data()[r + 1] || off.data()[r + 1] > data.size()) {
                                throw py::value_error("validate_context: entity seg off out of range");
                            }
                        }
                        seg_base.push_back(int64_t(D.arena.size()));
                        D.arena.insert(D.arena.end(), data.data(), data.data() + data.size());
                        seg_off.push_back(off);
                    }
                }
                // records of constrained DOFs only: a wire of Free DOFs (every
                // structured interior) allocates none
                if (tag != 0 && D.eparams.empty()) { D.eparams.assign(size_t(d.ndof) * EGG_B200_ENTITY_FIELDS, 0.0); }
                if (tag == EGG_B200_TAG_BSPLINE && seg_off.size() < 2) {
                    throw py::value_error("validate_context: a B-spline partition needs its knots and ctrl seg fields");
                }
                if (tag == EGG_B200_TAG_COMPOSITE && seg_off.empty()) {
                    throw py::value_error("validate_context: a composite partition needs its arena seg field");
                }
                if (tag == EGG_B200_TAG_BSPLINESURF && seg_off.size() < 3) {
                    throw py::value_error(
                      "validate_context: a B-spline surface partition needs its knots_u, knots_v and ctrl seg fields");
                }
                for (py::ssize_t i = 0; i < dl.size(); ++i) {
                    const int32_t v = dl.data()[i];
                    if (v < 0 || v >= d.ndof) { throw py::value_error("validate_context: dof_local out of range"); }
                    if (D.tags[v] != -1) { throw py::value_error("validate_context: dof_local covered by more than one SoA partition"); }
                    D.tags[v] = tag;
                    if (tag == 0) { continue; }
                    constrained = true;
                    // row i of the partition's (count, kFields) records
                    double* er = &D.eparams[size_t(v) * EGG_B200_ENTITY_FIELDS];
                    for (int f = 0; f < std::min(kf, int(EGG_B200_ENTITY_FIELDS)); ++f) { er[f] = rec.data()[i * kf + f]; }
                    if (tag == EGG_B200_TAG_BSPLINE) {
                        for (size_t k = 0; k < 3 && k < seg_off.size(); ++k) {
                            er[6 + k] = double(seg_base[k] + seg_off[k].data()[i]);
                        }
                    }
                    if (tag == EGG_B200_TAG_COMPOSITE && !seg_off.empty()) {  // the entity's arena slice
                        er[6] = double(seg_base[0] + seg_off[0].data()[i]);
                    }
                    if (tag == EGG_B200_TAG_BSPLINESURF) {
                        // knots_u, knots_v, ctrl, weights by arena offset; the UV
                        // trim (vertices, loop offsets) through a header
                        for (size_t k = 0; k < 4 && k < seg_off.size(); ++k) {
                            er[4 + k] = double(seg_base[k] + seg_off[k].data()[i]);
                        }
                        er[9] = -1.0;
                        if (seg_off.size() >= 6) {
                            const int64_t nl = seg_off[5].data()[i + 1] - seg_off[5].data()[i];
                            if (nl >= 2) {
                                er[9] = double(D.arena.size());
                                D.arena.push_back(double(nl));
                                D.arena.push_back(double(seg_base[5] + seg_off[5].data()[i]));
                                D.arena.push_back(double(seg_base[4] + seg_off[4].data()[i]));
                            }
                        }
                    }
                }
            }
            for (int64_t i = 0; i < d.ndof; ++i) {
                if (D.tags[i] == -1) {
                    throw py::value_error("validate_context: group[0] DOF " + std::to_string(i) + " not covered by any SoA partition");
                }
            }
        } else {
            std::fill(D.tags.begin(), D.tags.end(), 0);
        }
        d.entity_tag = D.tags.data();
        d.entity_params = constrained ? D.eparams.data() : nullptr;
        d.entity_arena = D.arena.empty() ? nullptr : D.arena.data();
        d.entity_arena_len = int64_t(D.arena.size());
        // Soft terms (src/bindings.cpp:380-410): per-DOF fixed-K tables with
        // global node ids; the core remaps them to owner slots.
        auto sized = [&](const char* key, int64_t want, bool real) -> const void* {
            int64_t got = 0;
            const void* ptr = real ? static_cast<const void*>(D.keep.reals(g[key], &got))
                                   : static_cast<const void*>(D.keep.ints(g[key], &got));
            if (got != want) {
                throw py::value_error(std::string("validate_context: group[0] ") + key + " size " + std::to_string(got) +
                                      " != " + std::to_string(want));
            }
            return ptr;
        };
        if (g.contains("curv_k")) {
            const int k = g["curv_k"].cast<int>();
            if (k < 0) { throw py::value_error("validate_context: group[0] curv_k < 0"); }
            if (k > 0) {
                d.curv_k = k;
                d.curv_nodes = static_cast<const int32_t*>(sized("curv_nodes", d.ndof * k * 4, false));
                d.curv_slot = static_cast<const int32_t*>(sized("curv_slot", d.ndof * k, false));
                d.curv_weight = static_cast<const double*>(sized("curv_weight", d.ndof * k, true));
            }
        }
        if (g.contains("dir_k")) {
            const int k = g["dir_k"].cast<int>();
            if (k < 0) { throw py::value_error("validate_context: group[0] dir_k < 0"); }
            if (k > 0) {
                d.dir_k = k;
                d.dir_eps = g["dir_eps"].cast<double>();
                d.dir_nodes = static_cast<const int32_t*>(sized("dir_nodes", d.ndof * k * 4, false));
                d.dir_slot = static_cast<const int32_t*>(sized("dir_slot", d.ndof * k, false));
                d.dir_kind = static_cast<const int32_t*>(sized("dir_kind", d.ndof * k, false));
                d.dir_ref = static_cast<const double*>(sized("dir_ref", d.ndof * k * dim, true));
                d.dir_weight = static_cast<const double*>(sized("dir_weight", d.ndof * k, true));
                // dir_axis (the 3D-only kinds' projector) is read by no kind yet
                if (g.contains("dir_axis")) { sized("dir_axis", d.ndof * k * dim, true); }
            }
        }
    }

    py::dict es = ctx["energy_stencil"].cast<py::dict>();
    d.es_num_samples = es["num_samples"].cast<int64_t>();
    d.es_structured = es.contains("structured") ? es["structured"].cast<int>() : 0;
    if (!d.es_structured) {
        int64_t n = 0;
        d.es_gc = D.keep.ints(es["gc"], &n);
        if (n != d.es_num_samples) { throw py::value_error("validate_context: energy_stencil gc size mismatch"); }
        for (int k = 0; k < dim; ++k) {
            d.es_gn[k] = D.keep.ints(es[("gn" + std::to_string(k)).c_str()], &n);
            if (n != d.es_num_samples) { throw py::value_error("validate_context: energy_stencil gn size mismatch"); }
            d.es_s[k] = D.keep.reals(es[("s" + std::to_string(k)).c_str()], &n);
            if (n != d.es_num_samples) { throw py::value_error("validate_context: energy_stencil s size mismatch"); }
        }
    }
    d.es_W_inv = D.keep.reals(es["W_inv"], &d.es_W_inv_len);
    if (es.contains("weight")) { d.es_weight = D.keep.reals(es["weight"], &d.es_weight_len); }
    // Whole-sample directional table (src/bindings.cpp:471-480).
    if (es.contains("dir_num") && es["dir_num"].cast<int64_t>() > 0) {
        const int64_t nd = es["dir_num"].cast<int64_t>();
        d.es_dir_num = nd;
        d.es_dir_eps = es["dir_eps"].cast<double>();
        int64_t n = 0;
        d.es_dir_nodes = D.keep.ints(es["dir_nodes"], &n);
        if (n != nd * 4) { throw py::value_error("validate_context: energy_stencil dir_nodes size mismatch"); }
        d.es_dir_kind = D.keep.ints(es["dir_kind"], &n);
        if (n != nd) { throw py::value_error("validate_context: energy_stencil dir_kind size mismatch"); }
        d.es_dir_ref = D.keep.reals(es["dir_ref"], &n);
        if (n != nd * dim) { throw py::value_error("validate_context: energy_stencil dir_ref size mismatch"); }
        d.es_dir_weight = D.keep.reals(es["dir_weight"], &n);
        if (n != nd) { throw py::value_error("validate_context: energy_stencil dir_weight size mismatch"); }
    }
}

py::array_t<double> vec(const std::vector<double>& v)
{
    py::array_t<double> out(py::ssize_t(v.size()));
    std::copy(v.begin(), v.end(), out.mutable_data());
    return out;
}

// The reference's single-block control wire (egg/smoothing/control_backend.py
// build_control_wire) -> egg_b200_control_desc.
void fill_control(egg_b200_control_desc& c, Keep& keep, const py::dict& w, int dim)
{
    if (w.contains("blocks")) {
        PyErr_SetString(PyExc_NotImplementedError,
                        "egg_b200: a multi-block control topology (control['blocks']) attaches to one "
                        "CppStructuredSweepSession; a batch takes one single-block net per mesh");
        throw py::error_already_set();
    }
    for (const char* k : {"block", "ctrl_shape", "k_supp", "C0", "free_idx", "b"}) {
        if (!w.contains(k)) { throw py::value_error(std::string("control: missing key '") + k + "'"); }
    }
    c = egg_b200_control_desc {};
    c.block = w["block"].cast<int32_t>();
    c.k_supp = w["k_supp"].cast<int32_t>();
    int64_t ncs = 0;
    const int32_t* cs = keep.ints(w["ctrl_shape"], &ncs);
    if (ncs != dim) { throw py::value_error("control: ctrl_shape must have D entries"); }
    for (int k = 0; k < dim; ++k) {
        c.ctrl_shape[k] = cs[k];
        const std::string ok = "off" + std::to_string(k), wk = "wt" + std::to_string(k);
        if (!w.contains(ok.c_str()) || !w.contains(wk.c_str())) {
            throw py::value_error("control: missing per-axis basis table " + ok + "/" + wk);
        }
        int64_t nw = 0;
        c.off[k] = keep.ints(w[ok.c_str()], &c.off_len[k]);
        c.wt[k] = keep.reals(w[wk.c_str()], &nw);
        if (nw != c.off_len[k] * int64_t(c.k_supp)) {
            throw py::value_error("control: wt" + std::to_string(k) + " size != off size * k_supp");
        }
    }
    int64_t nC = 0;
    c.C0 = keep.reals(w["C0"], &nC);
    int64_t nctrl = 1;
    for (int k = 0; k < dim; ++k) { nctrl *= c.ctrl_shape[k]; }
    if (nC != nctrl * dim) { throw py::value_error("control: C0 size != prod(ctrl_shape) * D"); }
    c.free_idx = keep.ints(w["free_idx"], &c.n_free);
    c.b = keep.reals(w["b"], &c.b_len);
}

// The reference's multi-block control wire (src/bindings.cpp:596-690
// unpack_control_topo, built by egg/smoothing/control_backend.py
// run_control_topo) -> egg_b200_control_topo_desc.  Per-block X0 (used only
// by the sliding-wall frames) is checked for size and otherwise unused.
struct TopoWire {
    std::vector<egg_b200_control_desc> nets;
    std::vector<double> arena;                  // the wire's arena plus B-spline-surface trim headers
    std::vector<std::vector<double>> surf_rec;  // converted B-spline-surface records
    std::vector<egg_b200_control_slide> slide;
    std::vector<egg_b200_control_wall_face> wall_faces;
    std::vector<int32_t> seam;
    std::vector<double> X0;
    egg_b200_control_topo_desc d {};
};

// The sliding-wall frame wire of a topology (src/bindings.cpp:681-722,
// egg/smoothing/control_backend.py:472-560): sliding roots, CAD wall faces,
// per-net seam flags, the entity arena and every net's X0.
void fill_topo_slides(TopoWire& t, Keep& keep, const py::dict& w, int dim, const std::vector<int64_t>& n_nodes)
{
    if (w.contains("arena")) {
        int64_t na = 0;
        const double* a = keep.reals(w["arena"], &na);
        t.arena.assign(a, a + na);
    }
    // A 3D B-spline surface blob (pu, pv, nu, nv, ku_off, kv_off, ctrl_off,
    // w_off, has_w, trim_v_off, trim_l_off, n_trim_loop_entries;
    // egg/smoothing/control_backend.py _encode_frame_entity) becomes this
    // core's record, its trim reached through a header in the arena.
    auto record = [&](int tag, const double* params, int64_t& len) -> const double* {
        if (dim != 3 || tag != EGG_B200_TAG_BSPLINESURF) { return params; }
        if (len < 9) { throw py::value_error("control topo: B-spline surface blob too short"); }
        std::vector<double> r(EGG_B200_ENTITY_FIELDS, 0.0);
        for (int k = 0; k < 9; ++k) { r[size_t(k)] = params[k]; }
        r[9] = -1.0;
        if (len >= 12 && params[11] >= 2) {
            r[9] = double(t.arena.size());
            t.arena.push_back(params[11]);
            t.arena.push_back(params[10]);
            t.arena.push_back(params[9]);
        }
        t.surf_rec.push_back(std::move(r));  // moving the outer vector keeps each record's buffer
        len = EGG_B200_ENTITY_FIELDS;
        return t.surf_rec.back().data();
    };
    for (const py::handle item : w["slide"].cast<py::list>()) {
        const py::dict sd = item.cast<py::dict>();
        egg_b200_control_slide r {};
        r.rep_row = sd["rep_row"].cast<int32_t>();
        int64_t nc = 0, nk = 0, ncomp = 0, nb = 0;
        r.members = keep.ints(sd["members"], &r.n_members);
        r.member_coef = keep.reals(sd["member_coef"], &nc);
        r.tag = sd["tag"].cast<int32_t>();
        r.params = keep.reals(sd["params"], &r.params_len);
        r.params = record(r.tag, r.params, r.params_len);
        r.r_entry = keep.ints(sd["r_entry"], &r.n_entries);
        r.comp = keep.ints(sd["comp"], &ncomp);
        r.kt = keep.ints(sd["kt"], &nk);
        r.base = keep.reals(sd["base"], &nb);
        if (nc != r.n_members || ncomp != r.n_entries || nk != r.n_entries || nb != r.n_entries) {
            throw py::value_error("control topo: slide list length mismatch");
        }
        t.slide.push_back(r);
    }
    for (const py::handle item : w["wall_faces"].cast<py::list>()) {
        const py::dict wd = item.cast<py::dict>();
        egg_b200_control_wall_face f {};
        f.net = wd["block"].cast<int32_t>();
        f.axis = wd["axis"].cast<int32_t>();
        f.side = wd["side"].cast<int32_t>();
        f.tag = wd["tag"].cast<int32_t>();
        f.params = keep.reals(wd["params"], &f.params_len);
        f.params = record(f.tag, f.params, f.params_len);
        t.wall_faces.push_back(f);
    }
    const py::list seams = w["seam_face"].cast<py::list>();
    if (size_t(py::len(seams)) != t.nets.size()) {
        throw py::value_error("control topo: seam_face flags must cover every net");
    }
    for (const py::handle item : seams) {
        int64_t nf = 0;
        const int32_t* fl = keep.ints(item, &nf);
        if (nf != 2 * dim) { throw py::value_error("control topo: seam_face flags must have 2*D entries"); }
        for (int64_t k = 0; k < nf; ++k) { t.seam.push_back(fl[k] != 0 ? 1 : 0); }
    }
    const py::list blocks = w["blocks"].cast<py::list>();
    for (size_t i = 0; i < t.nets.size(); ++i) {
        const py::dict bd = blocks[i].cast<py::dict>();
        if (!bd.contains("X0")) { throw py::value_error("control topo: the slide wire requires per-block X0"); }
        int64_t nx = 0;
        const double* x0 = keep.reals(bd["X0"], &nx);
        if (nx != n_nodes[i] * dim) { throw py::value_error("control topo: X0 size != prod(node_shape) * D"); }
        t.X0.insert(t.X0.end(), x0, x0 + nx);
    }
    t.d.n_slide = int32_t(t.slide.size());
    t.d.n_wall_faces = int32_t(t.wall_faces.size());
    t.d.slide = t.slide.data();
    t.d.wall_faces = t.wall_faces.data();
    t.d.seam_face = t.seam.data();
    t.d.X0 = t.X0.data();
    t.d.X0_len = int64_t(t.X0.size());
    t.d.arena = t.arena.empty() ? nullptr : t.arena.data();
    t.d.arena_len = int64_t(t.arena.size());
}

void fill_control_topo(TopoWire& t, Keep& keep, const py::dict& w, int dim)
{
    int64_t n_stack = 0;
    std::vector<int64_t> net_nodes;
    for (const py::handle item : w["blocks"].cast<py::list>()) {
        const py::dict bd = item.cast<py::dict>();
        egg_b200_control_desc c {};
        c.block = bd["block"].cast<int32_t>();
        int64_t ncs = 0;
        const int32_t* cs = keep.ints(bd["ctrl_shape"], &ncs);
        if (ncs != dim) { throw py::value_error("control topo: ctrl_shape must have D entries"); }
        int64_t n_ctrl = 1, n_nodes = 1;
        for (int k = 0; k < dim; ++k) {
            c.ctrl_shape[k] = cs[k];
            if (cs[k] < 2) { throw py::value_error("control topo: each ctrl_shape entry must be >= 2"); }
            n_ctrl *= cs[k];
        }
        c.k_supp = bd["k_supp"].cast<int32_t>();
        if (c.k_supp < 1) { throw py::value_error("control topo: k_supp must be >= 1"); }
        for (int k = 0; k < dim; ++k) {
            const std::string ok = "off" + std::to_string(k), wk = "wt" + std::to_string(k);
            int64_t nw = 0;
            c.off[k] = keep.ints(bd[ok.c_str()], &c.off_len[k]);
            c.wt[k] = keep.reals(bd[wk.c_str()], &nw);
            if (nw != c.off_len[k] * int64_t(c.k_supp)) {
                throw py::value_error("control topo: wt" + std::to_string(k) + " size != off size * k_supp");
            }
            for (int64_t i = 0; i < c.off_len[k]; ++i) {
                if (c.off[k][i] < 0 || c.off[k][i] + c.k_supp > c.ctrl_shape[k]) {
                    throw py::value_error("control topo: off" + std::to_string(k) +
                                          " support window out of the control lattice");
                }
            }
            n_nodes *= c.off_len[k];
        }
        c.b = keep.reals(bd["b"], &c.b_len);
        if (c.b_len != n_nodes * dim) { throw py::value_error("control topo: b size != prod(node_shape) * D"); }
        if (bd.contains("X0")) {
            int64_t nx = 0;
            keep.reals(bd["X0"], &nx);
            if (nx != n_nodes * dim) { throw py::value_error("control topo: X0 size != prod(node_shape) * D"); }
        }
        n_stack += n_ctrl;
        net_nodes.push_back(n_nodes);
        t.nets.push_back(c);
    }
    egg_b200_control_topo_desc& d = t.d;
    d = egg_b200_control_topo_desc {};
    d.n_nets = int32_t(t.nets.size());
    d.nets = t.nets.data();
    d.C0 = keep.reals(w["C0"], &d.C0_len);
    if (d.C0_len != n_stack * dim) { throw py::value_error("control topo: C0 size != total controls * D"); }
    d.nq = w["nq"].cast<int64_t>();
    int64_t ncol = 0;
    d.r_off = keep.ints(w["r_off"], &d.r_off_len);
    d.r_col = keep.ints(w["r_col"], &ncol);
    d.r_coef = keep.reals(w["r_coef"], &d.r_nnz);
    if (d.r_off_len != n_stack * dim + 1 || ncol != d.r_nnz || d.r_off[d.r_off_len - 1] != ncol) {
        throw py::value_error("control topo: malformed reduction CSR");
    }
    if (w.contains("p_off")) {
        int64_t pcol = 0;
        d.p_off = keep.ints(w["p_off"], &d.p_off_len);
        d.p_col = keep.ints(w["p_col"], &pcol);
        d.p_coef = keep.reals(w["p_coef"], &d.p_nnz);
        d.p_w = keep.reals(w["p_w"], &d.p_w_len);
        if (pcol != d.p_nnz || (d.p_off_len == 0 ? pcol != 0 : d.p_off[d.p_off_len - 1] != pcol) ||
            (d.p_off_len != 0 && d.p_w_len != d.p_off_len - 1)) {
            throw py::value_error("control topo: malformed penalty CSR");
        }
    }
    if (w.contains("slide")) { fill_topo_slides(t, keep, w, dim, net_nodes); }
}

// The walls of a single-block control wire (src/bindings.cpp:557-590): the
// exact node field X0 and one record per wall face.
struct WallWire {
    std::vector<egg_b200_control_wall> walls;
    const double* X0 = nullptr;
    int64_t X0_len = 0;
    bool present = false;
};

void fill_walls(WallWire& ww, Keep& keep, const py::dict& w, const egg_b200_control_desc& c, int dim)
{
    if (!w.contains("walls")) { return; }
    ww.present = true;
    if (!w.contains("X0")) { throw py::value_error("control: walls require X0"); }
    ww.X0 = keep.reals(w["X0"], &ww.X0_len);
    int64_t n_nodes = 1;
    for (int k = 0; k < dim; ++k) { n_nodes *= c.off_len[k]; }
    if (ww.X0_len != n_nodes * dim) { throw py::value_error("control: X0 size != prod(node_shape) * D"); }
    int64_t n_ctrl = 1;
    for (int k = 0; k < dim; ++k) { n_ctrl *= c.ctrl_shape[k]; }
    for (const py::handle item : w["walls"].cast<py::list>()) {
        const py::dict wd = item.cast<py::dict>();
        egg_b200_control_wall x {};
        x.axis = wd["axis"].cast<int32_t>();
        x.side = wd["side"].cast<int32_t>();
        x.mode = wd["mode"].cast<int32_t>();
        if (x.axis < 0 || x.axis >= dim || (x.side != 0 && x.side != 1) || x.mode < 0 || x.mode > 2) {
            throw py::value_error("control: wall axis/side/mode out of range");
        }
        int64_t nw = 0, n0 = 0, n1 = 0;
        x.weight = keep.reals(wd["weight"], &nw);
        x.p0 = keep.ints(wd["p0"], &n0);
        x.p1 = keep.ints(wd["p1"], &n1);
        if (n0 != n1 || nw != n0) { throw py::value_error("control: wall p0/p1/weight length mismatch"); }
        x.n_legs = n0;
        for (int64_t j = 0; j < n0; ++j) {
            if (x.p0[j] < 0 || x.p0[j] >= n_ctrl || x.p1[j] < 0 || x.p1[j] >= n_ctrl) {
                throw py::value_error("control: wall control id out of range");
            }
        }
        x.tag = wd["tag"].cast<int32_t>();
        x.params = keep.reals(wd["params"], &x.params_len);
        ww.walls.push_back(x);
    }
}

py::dict control_report(int n_outer, const std::vector<double>& E, const std::vector<double>& M,
                        const std::vector<double>& A, const std::vector<double>& PI, const std::vector<double>& PR,
                        const int64_t* cnt, int32_t iters, int32_t conv)
{
    auto take = [](const std::vector<double>& v, int64_t off, int64_t n) {
        return std::vector<double>(v.begin() + off, v.begin() + off + n);
    };
    (void)n_outer;
    py::dict out;
    out["energies"] = vec(take(E, 0, cnt[0]));
    out["mindets"] = vec(take(M, 0, cnt[0]));
    out["alphas"] = vec(take(A, 0, cnt[1]));
    out["pcg_iters"] = vec(take(PI, 0, cnt[2]));
    out["pcg_relres"] = vec(take(PR, 0, cnt[2]));
    out["frame_jumps"] = vec(std::vector<double>());
    out["iters"] = iters;
    out["converged"] = bool(conv);
    return out;
}

class Session
{
  public:
    Session(const py::dict& ctx, const py::dict& st, const DArr& X, const std::string& device, int dim,
            const py::object& control, const py::object& precision) :
        dim_(dim)
    {
        Desc D;
        fill_desc(D, ctx, st, X, dim, parse_precision(precision), device_of(device));
        Keep ckeep;
        egg_b200_control_desc cdesc;
        TopoWire topo;
        WallWire walls;
        const bool is_topo = !control.is_none() && control.cast<py::dict>().contains("blocks");
        if (is_topo) {
            fill_control_topo(topo, ckeep, control.cast<py::dict>(), dim);
        } else if (!control.is_none()) {
            fill_control(cdesc, ckeep, control.cast<py::dict>(), dim);
            fill_walls(walls, ckeep, control.cast<py::dict>(), cdesc, dim);
        }
        egg_b200_session* h = nullptr;
        {
            py::gil_scoped_release nogil;
            const int rc = egg_b200_session_create(&D.d, &h);
            if (rc != EGG_B200_OK) {
                py::gil_scoped_acquire g;
                raise_status(rc);
            }
        }
        h_.reset(h);
        M_ = D.d.num_nodes;
        nblocks_ = D.d.num_blocks;
        if (is_topo) {
            check(egg_b200_session_attach_control_topo(h_.get(), &topo.d));
        } else if (!walls.walls.empty()) {
            check(egg_b200_session_attach_control_walls(h_.get(), &cdesc, walls.X0, walls.X0_len,
                                                        int32_t(walls.walls.size()), walls.walls.data()));
        } else if (!control.is_none()) {
            check(egg_b200_session_attach_control(h_.get(), &cdesc));
        }
    }

    void set_control_reduction(int64_t nq, const IArr& off, const IArr& col, const DArr& coef)
    {
        if (col.size() != coef.size()) { throw py::value_error("control topo: malformed reduction CSR"); }
        check(egg_b200_session_set_control_reduction(h_.get(), nq, off.data(), int64_t(off.size()), col.data(),
                                                     coef.data(), int64_t(coef.size())));
    }

    void set_control_penalty(const IArr& off, const IArr& col, const DArr& coef, const DArr& w)
    {
        if (col.size() != coef.size()) { throw py::value_error("control topo: malformed penalty CSR"); }
        check(egg_b200_session_set_control_penalty(h_.get(), off.data(), int64_t(off.size()), col.data(), coef.data(),
                                                   int64_t(coef.size()), w.data(), int64_t(w.size())));
    }

    void set_control_b(int block_index, const DArr& b)
    {
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = egg_b200_session_set_control_b(h_.get(), block_index, b.data(), int64_t(b.size()));
        }
        check(rc);
    }

    py::dict run_control(int n_outer, const std::string& phase, double grad_tol, double alpha_min, double lm0,
                         int pcg_max_iter, double pcg_rtol, bool pcg_forcing, bool model_db)
    {
        const int64_t ce = int64_t(n_outer) + 1, ca = std::max(n_outer, 1), cp = 8 * ca;
        std::vector<double> E(static_cast<size_t>(ce)), M(static_cast<size_t>(ce)), A(static_cast<size_t>(ca));
        std::vector<double> PI(static_cast<size_t>(cp)), PR(static_cast<size_t>(cp)), FJ(static_cast<size_t>(ca));
        int64_t cnt[3] = {0, 0, 0}, nfj = 0;
        int32_t iters = 0, conv = 0;
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = egg_b200_session_run_control_ex(h_.get(), n_outer, objective_of(phase), grad_tol, alpha_min, lm0,
                                                 pcg_max_iter, pcg_rtol, pcg_forcing ? 1 : 0, model_db ? 1 : 0,
                                                 E.data(), M.data(), A.data(), PI.data(), PR.data(), cnt, &iters,
                                                 &conv, FJ.data(), &nfj);
        }
        check(rc);
        py::dict out = control_report(n_outer, E, M, A, PI, PR, cnt, iters, conv);
        FJ.resize(static_cast<size_t>(nfj));
        out["frame_jumps"] = vec(FJ);
        return out;
    }

    py::array_t<double> get_C()
    {
        int64_t n = 0;
        check(egg_b200_session_control_size(h_.get(), &n));
        if (n == 0) { throw py::value_error("get_C: session has no control wire"); }
        std::vector<double> C(static_cast<size_t>(n));
        check(egg_b200_session_get_C(h_.get(), C.data(), n));
        return vec(C);
    }

    void set_C(const DArr& C)
    {
        int64_t n = 0;
        check(egg_b200_session_control_size(h_.get(), &n));
        if (n == 0) { throw py::value_error("set_C: session has no control wire"); }
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = egg_b200_session_set_C(h_.get(), C.data(), int64_t(C.size()));
        }
        check(rc);
    }

    std::tuple<py::array_t<double>, py::array_t<double>> run(int n_sweeps, const std::string& phase, double delta,
                                                             double omega, int report_every)
    {
        const int k = report_every <= 0 ? std::max(n_sweeps, 1) : report_every;
        const int64_t cap = n_sweeps > 0 ? (int64_t(n_sweeps) + k - 1) / k : 0;
        std::vector<double> E(static_cast<size_t>(cap)), Md(static_cast<size_t>(cap));
        int64_t nrep = 0;
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = egg_b200_session_run(h_.get(), n_sweeps, objective_of(phase), delta, omega, report_every, E.data(),
                                      Md.data(), cap, &nrep);
        }
        check(rc);
        E.resize(size_t(nrep));
        Md.resize(size_t(nrep));
        return {vec(E), vec(Md)};
    }

    std::tuple<py::array_t<double>, py::array_t<double>> run_fas(int n_cycles, int nu_pre, int nu_post,
                                                                 int nu_coarse, double omega, int max_levels,
                                                                 const std::string& phase)
    {
        const int per = std::max(nu_pre + nu_post, 1);
        const int64_t cap = std::max<int64_t>(int64_t(n_cycles) * per, 1);
        std::vector<double> E(static_cast<size_t>(cap)), Md(static_cast<size_t>(cap));
        int64_t nrep = 0;
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = egg_b200_session_run_fas(h_.get(), n_cycles, nu_pre, nu_post, nu_coarse, omega, max_levels,
                                          objective_of(phase), E.data(), Md.data(), cap, &nrep);
        }
        check(rc);
        E.resize(size_t(nrep));
        Md.resize(size_t(nrep));
        return {vec(E), vec(Md)};
    }

    py::list mg_levels()
    {
        int32_t n = 0;
        check(egg_b200_session_mg_levels(h_.get(), &n));
        py::list levels;
        for (int32_t l = 0; l < n; ++l) {
            std::vector<int32_t> sh(size_t(nblocks_) * dim_);
            check(egg_b200_session_mg_level_shapes(h_.get(), l, sh.data(), int64_t(sh.size())));
            py::list blocks;
            for (int b = 0; b < nblocks_; ++b) {
                py::tuple t(dim_);
                for (int k = 0; k < dim_; ++k) { t[k] = sh[size_t(b) * dim_ + k]; }
                blocks.append(t);
            }
            levels.append(blocks);
        }
        return levels;
    }

    py::array_t<double> get_X()
    {
        // A page-locked buffer from the pool when one can be had, so the
        // device writes straight into the result; it returns to the pool when
        // the array is freed.  Otherwise ordinary numpy memory.
        const int64_t n = int64_t(M_ * dim_), bytes = n * int64_t(sizeof(double));
        void* pin = nullptr;
        py::array_t<double> X;
        if (bytes > 0 && egg_b200_pinned_acquire(bytes, &pin) == EGG_B200_OK && pin) {
            auto* rec = new PinnedBuf {pin, bytes};
            py::capsule owner(rec, [](void* r) {
                auto* b = static_cast<PinnedBuf*>(r);
                egg_b200_pinned_release(b->p);
                delete b;
            });
            X = py::array_t<double>({py::ssize_t(n)}, {py::ssize_t(sizeof(double))}, static_cast<double*>(pin), owner);
        } else {
            X = py::array_t<double>(py::ssize_t(n));
        }
        double* out = X.mutable_data();
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = egg_b200_session_get_X(h_.get(), out, int64_t(M_ * dim_));
        }
        check(rc);
        return X;
    }

    void set_X(const DArr& X)
    {
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = egg_b200_session_set_X(h_.get(), X.data(), int64_t(X.size()));
        }
        check(rc);
    }

    std::tuple<double, double> energy(const std::string& phase, double delta)
    {
        double e = 0, m = 0;
        check(egg_b200_session_energy(h_.get(), objective_of(phase), delta, &e, &m));
        return {e, m};
    }

    std::tuple<double, double> energy_noalloc(const std::string& phase, double delta, int n_partials)
    {
        double e = 0, m = 0;
        check(egg_b200_session_energy_noalloc(h_.get(), objective_of(phase), delta, n_partials, &e, &m));
        return {e, m};
    }

    py::dict info()
    {
        int64_t v[11];
        check(egg_b200_session_info(h_.get(), v, 11));
        py::dict d;
        const char* keys[11] = {"dim",    "num_nodes",      "store_nodes",       "ndof",      "interior_dofs", "stored_dofs",
                                "copies", "energy_samples", "structured_energy", "precision", "updates"};
        for (int i = 0; i < 11; ++i) { d[keys[i]] = v[i]; }
        d["precision"] = v[9] == EGG_B200_PREC_MIXED ? "mixed" : "fp64";
        return d;
    }

    void set_profiling(bool on) { check(egg_b200_session_set_profiling(h_.get(), on ? 1 : 0)); }

    py::dict kernel_stats()
    {
        static const char* names[8] = {"interior_sweep", "stored_sweep", "broadcast",    "reduce",
                                       "reduce_final",   "copy",         "fas_transfer", "control"};
        py::dict d;
        for (int k = 0; k < 8; ++k) {
            double ms = 0;
            int64_t n = 0;
            check(egg_b200_session_kernel_stats(h_.get(), k, &ms, &n));
            d[names[k]] = py::make_tuple(ms, n);
        }
        return d;
    }

    void reset_stats() { check(egg_b200_session_reset_stats(h_.get())); }

    void checkpoint()
    {
        py::gil_scoped_release nogil;
        const int rc = egg_b200_session_checkpoint(h_.get());
        py::gil_scoped_acquire g;
        check(rc);
    }

    void restore()
    {
        py::gil_scoped_release nogil;
        const int rc = egg_b200_session_restore(h_.get());
        py::gil_scoped_acquire g;
        check(rc);
    }

    int autotune(const std::string& phase, int reps)
    {
        int32_t v = 0;
        py::gil_scoped_release nogil;
        const int rc = egg_b200_session_autotune(h_.get(), objective_of(phase), reps, &v);
        py::gil_scoped_acquire g;
        check(rc);
        return v;
    }

    void set_variant(int v) { check(egg_b200_session_set_variant(h_.get(), v)); }

    py::dict variants()
    {
        int32_t v = 0, shape[5 * EGG_B200_NUM_VARIANTS];
        double t[EGG_B200_NUM_VARIANTS];
        check(egg_b200_session_variant_info(h_.get(), &v, shape, t, EGG_B200_NUM_VARIANTS));
        py::dict d;
        d["variant"] = v;
        py::list lst;
        for (int i = 0; i < EGG_B200_NUM_VARIANTS; ++i) {
            lst.append(py::make_tuple(shape[5 * i], shape[5 * i + 1], shape[5 * i + 2], shape[5 * i + 3],
                                      shape[5 * i + 4], t[i]));
        }
        d["table"] = lst;
        return d;
    }

    uintptr_t stream()
    {
        void* p = nullptr;
        check(egg_b200_session_stream(h_.get(), &p));
        return reinterpret_cast<uintptr_t>(p);
    }

    int64_t launch_count()
    {
        int64_t n = 0;
        check(egg_b200_session_launch_count(h_.get(), &n));
        return n;
    }

  protected:
    explicit Session(int dim) : dim_(dim) {}
    struct Del {
        void operator()(egg_b200_session* s) const { egg_b200_session_destroy(s); }
    };
    int dim_;
    int nblocks_ = 0;
    int64_t M_ = 0;
    std::unique_ptr<egg_b200_session, Del> h_;
};

// Several independent meshes in one device-resident session (one launch per
// kernel over all meshes, per-mesh reports).
class Batch : public Session
{
  public:
    Batch(const py::sequence& meshes, const std::string& device, int dim, const py::object& precision,
          const py::object& control) :
        Session(dim)
    {
        const int prec = parse_precision(precision);
        const int dev = device_of(device);
        const size_t n = py::len(meshes);
        if (n == 0) { throw py::value_error("CppBatchSweepSession: no meshes"); }
        std::vector<Desc> descs(n);
        std::vector<egg_b200_session_desc> raw(n);
        for (size_t m = 0; m < n; ++m) {
            py::sequence t = meshes[m].cast<py::sequence>();
            if (py::len(t) != 3) { throw py::value_error("CppBatchSweepSession: each mesh is (ctx_arrays, structured, X)"); }
            fill_desc(descs[m], t[0].cast<py::dict>(), t[1].cast<py::dict>(), DArr::ensure(t[2]), dim, prec, dev);
            raw[m] = descs[m].d;
        }
        Keep ckeep;
        std::vector<egg_b200_control_desc> cds;
        if (!control.is_none()) {
            py::sequence cl = control.cast<py::sequence>();
            if (size_t(py::len(cl)) != n) { throw py::value_error("control: one wire per mesh is required"); }
            cds.resize(n);
            for (size_t m = 0; m < n; ++m) {
                const py::dict wm = cl[m].cast<py::dict>();
                if (wm.contains("walls") && py::len(wm["walls"]) > 0) {
                    PyErr_SetString(PyExc_NotImplementedError,
                                    "egg_b200: control walls attach to one CppStructuredSweepSession; a batch takes "
                                    "plain nets");
                    throw py::error_already_set();
                }
                fill_control(cds[m], ckeep, wm, dim);
            }
        }
        egg_b200_session* h = nullptr;
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = egg_b200_batch_create(raw.data(), int32_t(n), &h);
        }
        check(rc);
        h_.reset(h);
        int32_t nm = 0;
        offs_.resize(n + 1);
        check(egg_b200_batch_size(h_.get(), &nm, offs_.data()));
        n_ = nm;
        M_ = offs_.back();
        nblocks_ = 0;
        for (const auto& d : raw) { nblocks_ += d.num_blocks; }
        if (!cds.empty()) { check(egg_b200_batch_attach_controls(h_.get(), cds.data())); }
    }

    // One report dict per mesh.
    py::list run_control_batch(int n_outer, const std::string& phase, double grad_tol, double alpha_min, double lm0,
                               int pcg_max_iter, double pcg_rtol, bool pcg_forcing, bool model_db)
    {
        (void)model_db;
        const int64_t ce = int64_t(n_outer) + 1, ca = std::max(n_outer, 1), cp = 8 * ca;
        const size_t n = size_t(n_);
        std::vector<double> E(n * ce), M(n * ce), A(n * ca), PI(n * cp), PR(n * cp);
        std::vector<int64_t> cnt(3 * n);
        std::vector<int32_t> iters(n), conv(n);
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = egg_b200_batch_run_control(h_.get(), n_outer, objective_of(phase), grad_tol, alpha_min, lm0,
                                            pcg_max_iter, pcg_rtol, pcg_forcing ? 1 : 0, E.data(), M.data(), A.data(),
                                            PI.data(), PR.data(), cnt.data(), iters.data(), conv.data());
        }
        check(rc);
        py::list out;
        for (size_t m = 0; m < n; ++m) {
            auto sl = [&](const std::vector<double>& v, int64_t stride) {
                return std::vector<double>(v.begin() + int64_t(m) * stride, v.begin() + int64_t(m + 1) * stride);
            };
            out.append(control_report(n_outer, sl(E, ce), sl(M, ce), sl(A, ca), sl(PI, cp), sl(PR, cp), &cnt[3 * m],
                                      iters[m], conv[m]));
        }
        return out;
    }

    int num_meshes() const { return n_; }

    std::vector<int64_t> node_offsets() const { return offs_; }

    // (energies, mindets) of shape (n_meshes, reports).
    std::tuple<py::array_t<double>, py::array_t<double>> run(int n_sweeps, const std::string& phase, double delta,
                                                             double omega, int report_every)
    {
        const int k = report_every <= 0 ? std::max(n_sweeps, 1) : report_every;
        const int64_t cap = n_sweeps > 0 ? (int64_t(n_sweeps) + k - 1) / k : 0;
        std::vector<double> E(static_cast<size_t>(cap * n_)), Md(static_cast<size_t>(cap * n_));
        int64_t nrep = 0;
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = egg_b200_batch_run(h_.get(), n_sweeps, objective_of(phase), delta, omega, report_every, E.data(),
                                    Md.data(), cap, &nrep);
        }
        check(rc);
        py::array_t<double> e({int64_t(n_), nrep}), md({int64_t(n_), nrep});
        auto ev = e.mutable_unchecked<2>();
        auto mv = md.mutable_unchecked<2>();
        for (int64_t r = 0; r < nrep; ++r) {
            for (int m = 0; m < n_; ++m) {
                ev(m, r) = E[size_t(r * n_ + m)];
                mv(m, r) = Md[size_t(r * n_ + m)];
            }
        }
        return {e, md};
    }

    std::tuple<py::array_t<double>, py::array_t<double>> energy(const std::string& phase, double delta)
    {
        std::vector<double> E(static_cast<size_t>(n_)), Md(static_cast<size_t>(n_));
        check(egg_b200_batch_energy(h_.get(), objective_of(phase), delta, E.data(), Md.data()));
        return {vec(E), vec(Md)};
    }

    // Per-mesh positions (each flat, global node order of its mesh).
    py::list get_X_list()
    {
        py::array_t<double> all = get_X();
        const double* p = all.data();
        py::list out;
        for (int m = 0; m < n_; ++m) {
            std::vector<double> x(p + offs_[m] * dim_, p + offs_[m + 1] * dim_);
            out.append(vec(x));
        }
        return out;
    }

    void set_X_list(const py::sequence& Xs)
    {
        if (int(py::len(Xs)) != n_) { throw py::value_error("set_X: one array per mesh is required"); }
        std::vector<double> all(static_cast<size_t>(M_ * dim_));
        for (int m = 0; m < n_; ++m) {
            DArr a = DArr::ensure(Xs[m]);
            if (!a || int64_t(a.size()) != (offs_[m + 1] - offs_[m]) * dim_) {
                throw py::value_error("set_X: mesh " + std::to_string(m) + " has the wrong length");
            }
            std::copy(a.data(), a.data() + a.size(), all.begin() + offs_[m] * dim_);
        }
        set_X(DArr(py::array_t<double>(int64_t(all.size()), all.data())));
    }

  private:
    int n_ = 0;
    std::vector<int64_t> offs_;
};

}  // namespace

PYBIND11_MODULE(cpp_core, m)
{
    m.doc() = "egg compute core, B200 (sm_100a) CUDA build.";
    m.def("ping", [] { return 0; }, "Liveness check; returns 0.");
    // B-spline degree caps of the reference build (constrained boundaries are
    // not on this core's path; the values are kept for wire encoders).
    m.attr("MAX_BSPLINE_DEGREE") = 5;
    m.attr("MAX_BSPLINE_CURVE_DEGREE") = 7;
    m.attr("REAL_IS_FLOAT") = default_precision() == EGG_B200_PREC_MIXED;
    m.attr("ABI_VERSION") = egg_b200_abi_version();

    m.def("device_count", [] {
        int n = 0;
        check(egg_b200_device_count(&n));
        return n;
    });

    py::class_<Session>(m, "CppStructuredSweepSession",
                        "Persistent device-resident structured smoothing session (B200 CUDA core).")
      .def(py::init<py::dict, py::dict, DArr, const std::string&, int, const py::object&, const py::object&>(),
           py::arg("ctx_arrays"), py::arg("structured"), py::arg("X"), py::kw_only(), py::arg("device") = "auto",
           py::arg("dim") = 2, py::arg("control") = py::none(), py::arg("precision") = py::none())
      .def("run", &Session::run, py::arg("n_sweeps"), py::kw_only(), py::arg("phase") = "barrier",
           py::arg("delta") = 0.0, py::arg("omega") = 1.0, py::arg("report_every") = 0,
           "Run n_sweeps of block-Jacobi on the resident X; returns (energies, mindets).")
      .def("run_fas", &Session::run_fas, py::arg("n_cycles"), py::kw_only(), py::arg("nu_pre") = 2,
           py::arg("nu_post") = 2, py::arg("nu_coarse") = 32, py::arg("omega") = 1.0, py::arg("max_levels") = 32,
           py::arg("phase") = "barrier")
      .def("mg_levels", &Session::mg_levels)
      .def("get_X", &Session::get_X, "Download X gathered back to global node order, shape (N*dim,).")
      .def("set_X", &Session::set_X, py::arg("X"), "Upload X (global node order) into every copy.")
      .def("energy", &Session::energy, py::arg("phase") = "barrier", py::arg("delta") = 0.0,
           "(energy, min det A) of the resident state.")
      .def("energy_noalloc", &Session::energy_noalloc, py::arg("phase") = "barrier", py::arg("delta") = 0.0,
           py::arg("n_partials") = 0,
           "energy() through the allocation-free entry point (scratch in one static device array shared by all calls).")
      .def("info", &Session::info)
      .def("set_profiling", &Session::set_profiling, py::arg("enable"))
      .def("kernel_stats", &Session::kernel_stats)
      .def("reset_stats", &Session::reset_stats)
      .def("checkpoint", &Session::checkpoint, "Copy the resident positions to a device-side checkpoint.")
      .def("restore", &Session::restore, "Restore the resident positions from the device-side checkpoint.")
      .def("launch_count", &Session::launch_count)
      .def("stream", &Session::stream, "The session's cudaStream_t as an integer (for host-side events).")
      .def("autotune", &Session::autotune, py::arg("phase") = "barrier", py::arg("reps") = 3)
      .def("set_variant", &Session::set_variant, py::arg("variant"))
      .def("variants", &Session::variants)
      .def("run_control", &Session::run_control, py::arg("n_outer"), py::kw_only(), py::arg("phase") = "barrier",
           py::arg("grad_tol") = 1e-8, py::arg("alpha_min") = 1e-4, py::arg("lm0") = 0.0, py::arg("pcg_max_iter") = 200,
           py::arg("pcg_rtol") = 1e-10, py::arg("pcg_forcing") = true, py::arg("model_db") = true,
           "Damped reduced Gauss-Newton on the control net; returns the reference's report dict.")
      .def("get_C", &Session::get_C, "The resident control lattice, flat (n_ctrl * dim,).")
      .def("set_C", &Session::set_C, py::arg("C"), "Upload a control lattice and evaluate X = M C + b.")
      .def("set_control_reduction", &Session::set_control_reduction, py::arg("nq"), py::arg("off"), py::arg("col"),
           py::arg("coef"), "Replace the multi-block reduction CSR dC = R dq.")
      .def("set_control_penalty", &Session::set_control_penalty, py::arg("off"), py::arg("col"), py::arg("coef"),
           py::arg("w"), "Replace the multi-block penalty rows (1/2 sum_j w_j (P_j C)^2); empty off removes them.")
      .def("set_control_b", &Session::set_control_b, py::arg("block_index"), py::arg("b"),
           "Replace one net's Boolean-sum offset b and re-evaluate X.");

    py::class_<Batch, Session>(m, "CppBatchSweepSession",
                               "Several independent meshes swept together in one device-resident session.")
      .def(py::init<py::sequence, const std::string&, int, const py::object&, const py::object&>(), py::arg("meshes"),
           py::kw_only(), py::arg("device") = "auto", py::arg("dim") = 2, py::arg("precision") = py::none(),
           py::arg("control") = py::none(),
           "meshes: sequence of (ctx_arrays, structured, X) tuples, one per mesh; control: one wire per mesh or None.")
      .def("run_control", &Batch::run_control_batch, py::arg("n_outer"), py::kw_only(), py::arg("phase") = "barrier",
           py::arg("grad_tol") = 1e-8, py::arg("alpha_min") = 1e-4, py::arg("lm0") = 0.0, py::arg("pcg_max_iter") = 200,
           py::arg("pcg_rtol") = 1e-10, py::arg("pcg_forcing") = true, py::arg("model_db") = true,
           "run_control on every mesh's net together; one report dict per mesh.")
      .def_property_readonly("num_meshes", &Batch::num_meshes)
      .def("node_offsets", &Batch::node_offsets)
      .def("run", &Batch::run, py::arg("n_sweeps"), py::kw_only(), py::arg("phase") = "barrier",
           py::arg("delta") = 0.0, py::arg("omega") = 1.0, py::arg("report_every") = 0,
           "Run n_sweeps on every mesh; returns (energies, mindets) of shape (num_meshes, reports).")
      .def("energy", &Batch::energy, py::arg("phase") = "barrier", py::arg("delta") = 0.0,
           "Per-mesh (energies, mindets) of the resident state.")
      .def("get_X", &Batch::get_X_list, "Per-mesh positions, a list of flat arrays in each mesh's node order.")
      .def("set_X", &Batch::set_X_list, py::arg("X"), "Upload per-mesh positions (a list of flat arrays).");

    m.def(
      "cpp_structured_sweep",
      [](const py::dict& ctx, const py::dict& st, const DArr& X, int n_sweeps, const std::string& device,
         const std::string& phase, double delta, int dim, double omega, int report_every, const py::object& precision) {
          Session s(ctx, st, X, device, dim, py::none(), precision);
          auto [e, m] = s.run(n_sweeps, phase, delta, omega, report_every);
          return std::make_tuple(s.get_X(), e, m);
      },
      py::arg("ctx_arrays"), py::arg("structured"), py::arg("X"), py::arg("n_sweeps"), py::kw_only(),
      py::arg("device") = "auto", py::arg("phase") = "barrier", py::arg("delta") = 0.0, py::arg("dim") = 2,
      py::arg("omega") = 1.0, py::arg("report_every") = 0, py::arg("precision") = py::none(),
      "Run n_sweeps of block-Jacobi; returns (X_out, energies, mindets), X_out in global node order.");

    m.def(
      "metric_eval",
      [](const DArr& t, const std::string& metric, double delta) {
          int obj;
          if (metric == "shape_2d") {
              obj = EGG_B200_OBJ_SHAPE;
          } else if (metric == "shape_size") {
              obj = EGG_B200_OBJ_SHAPE_SIZE;
          } else if (metric == "untangle") {
              obj = EGG_B200_OBJ_UNTANGLE;
          } else {
              throw py::value_error("metric_eval: unknown metric '" + metric + "'");
          }
          if (t.size() != 4) { throw py::value_error("metric_eval: t must have 4 entries"); }
          double mu = 0;
          std::vector<double> g(4), h(16);
          check(egg_b200_metric_eval(obj, delta, t.data(), 1, &mu, g.data(), h.data()));
          return std::make_tuple(mu, vec(g), vec(h));
      },
      py::arg("t"), py::arg("metric") = "shape_2d", py::arg("delta") = 0.0,
      "Evaluate a named 2D metric on the GPU. Returns (mu, grad(4,), hess(16,)).");

    m.def(
      "metric_eval_3d",
      [](const DArr& t, const py::object& v_obj, const std::string& metric, double delta) {
          int obj = EGG_B200_OBJ_SHAPE;
          if (metric == "shape_size") {
              obj = EGG_B200_OBJ_SHAPE_SIZE;
          } else if (metric == "untangle") {
              obj = EGG_B200_OBJ_UNTANGLE;
          } else if (metric != "cond3" && metric != "shape") {
              throw py::value_error("metric_eval_3d: unknown metric '" + metric + "'");
          }
          if (t.size() != 9) { throw py::value_error("metric_eval_3d: t must have 9 entries"); }
          std::vector<double> v = {1.0, 1.0, 1.0};
          if (!v_obj.is_none()) {
              DArr va = DArr::ensure(v_obj);
              if (!va || va.size() != 3) { throw py::value_error("metric_eval_3d: v must have 3 entries"); }
              v.assign(va.data(), va.data() + 3);
          }
          double mu = 0;
          std::vector<double> g(9), hv(6);
          check(egg_b200_metric3_probe(obj, delta, t.data(), v.data(), 1, &mu, g.data(), hv.data()));
          return std::make_tuple(mu, vec(g), vec(hv));
      },
      py::arg("t"), py::arg("v") = py::none(), py::arg("metric") = "cond3", py::arg("delta") = 0.0,
      "3D metric on the GPU: (mu, grad over vec(T) (9,), contracted Hessian along e_i v^T packed (6,)).");

    m.def(
      "patch_eval",
      [](const DArr& X, const IArr& gc, const IArr& gn0, const IArr& gn1, const DArr& s0, const DArr& s1,
         const DArr& W, const IArr& role, const py::object&) {
          const int P = int(gc.size());
          if (gn0.size() != P || gn1.size() != P || s0.size() != P || s1.size() != P || role.size() != P ||
              W.size() != 4 * P) {
              throw py::value_error("patch_eval: inconsistent patch array sizes");
          }
          std::vector<double> g(2), h(4), st(2);
          double e = 0, md = 0;
          check(egg_b200_patch_eval(EGG_B200_OBJ_SHAPE, 0.0, X.data(), int64_t(X.size() / 2), P, gc.data(), gn0.data(),
                                    gn1.data(), s0.data(), s1.data(), W.data(), role.data(), g.data(), h.data(), &e,
                                    &md, st.data()));
          return std::make_tuple(vec(g), vec(h), e, md);
      },
      py::arg("X"), py::arg("gc"), py::arg("gn0"), py::arg("gn1"), py::arg("s0"), py::arg("s1"), py::arg("W_inv"),
      py::arg("role"), py::arg("J") = py::none(),
      "Per-DOF patch evaluation on the GPU. Returns (grad(2,), hess(4,), energy, mindet).");

    m.def(
      "newton_step",
      [](const DArr& grad, const DArr& hess, const DArr& pos, int tag, const py::object& params) {
          if (grad.size() != 2 || hess.size() != 4 || pos.size() != 2) {
              throw py::value_error("newton_step: grad(2), hess(4), pos(2) expected");
          }
          std::vector<double> x(2);
          if (tag == 0) {
              check(egg_b200_newton_step(grad.data(), hess.data(), x.data()));
              return vec(x);
          }
          if (params.is_none()) { throw py::value_error("newton_step: a constrained tag needs its params"); }
          DArr pr = DArr::ensure(params);
          std::vector<double> rec(EGG_B200_ENTITY_FIELDS, 0.0);
          for (py::ssize_t i = 0; i < std::min<py::ssize_t>(pr.size(), EGG_B200_ENTITY_FIELDS); ++i) {
              rec[size_t(i)] = pr.data()[i];
          }
          std::vector<double> foot(2);
          check(egg_b200_entity_step(tag, rec.data(), grad.data(), hess.data(), pos.data(), x.data(), foot.data()));
          return vec(x);
      },
      py::arg("grad"), py::arg("hess"), py::arg("pos"), py::arg("tag") = 0, py::arg("params") = py::none(),
      "Newton step: -H^{-1} g for a Free DOF (tag 0), or reduced onto the tangent of a 2D curve entity "
      "(LineSeg, Circle, Ellipse, LineRail; params = its record). Returns delta(2,).");

    m.def(
      "entity_project",
      [](const DArr& pos, int tag, const DArr& params) {
          if (pos.size() != 2) { throw py::value_error("entity_project: pos(2) expected"); }
          std::vector<double> rec(EGG_B200_ENTITY_FIELDS, 0.0);
          for (py::ssize_t i = 0; i < std::min<py::ssize_t>(params.size(), EGG_B200_ENTITY_FIELDS); ++i) {
              rec[size_t(i)] = params.data()[i];
          }
          const double g[2] = {0.0, 0.0}, h[4] = {1.0, 0.0, 0.0, 1.0};
          double st[2];
          std::vector<double> foot(2);
          check(egg_b200_entity_step(tag, rec.data(), g, h, pos.data(), st, foot.data()));
          return vec(foot);
      },
      py::arg("pos"), py::arg("tag"), py::arg("params"),
      "Projection of pos onto a 2D curve entity (device evaluation). Returns foot(2,).");

    // A 2D curve's record from its parameter blob, padded to the record width.
    auto record_of = [](const DArr& params) {
        std::vector<double> rec(EGG_B200_ENTITY_FIELDS, 0.0);
        for (py::ssize_t i = 0; i < std::min<py::ssize_t>(params.size(), EGG_B200_ENTITY_FIELDS); ++i) {
            rec[size_t(i)] = params.data()[i];
        }
        return rec;
    };
    m.def(
      "geometry_project",
      [record_of](const DArr& p, int tag, const DArr& params) {
          if (p.size() != 2) { throw py::value_error("geometry_project: p(2) expected"); }
          const std::vector<double> rec = record_of(params);
          std::vector<double> foot(2), tang(2);
          check(egg_b200_entity_frame(2, tag, rec.data(), nullptr, 0, p.data(), 1, foot.data(), tang.data()));
          return vec(foot);
      },
      py::arg("p"), py::arg("tag"), py::arg("params"), "Project point onto entity (device evaluation). Returns proj(2,).");
    m.def(
      "geometry_tangent",
      [record_of](const DArr& p, int tag, const DArr& params) {
          if (p.size() != 2) { throw py::value_error("geometry_tangent: p(2) expected"); }
          const std::vector<double> rec = record_of(params);
          std::vector<double> foot(2), tang(2);
          check(egg_b200_entity_frame(2, tag, rec.data(), nullptr, 0, p.data(), 1, foot.data(), tang.data()));
          return vec(tang);
      },
      py::arg("p"), py::arg("tag"), py::arg("params"),
      "Tangent direction at point on entity (device evaluation). Returns tang(2,).");
    m.def(
      "geometry_project_batch",
      [](const py::array_t<double, py::array::c_style | py::array::forcecast>& q, int tag, const DArr& records,
         const py::list& seg) {
          if (q.ndim() != 2 || (q.shape(1) != 2 && q.shape(1) != 3)) {
              throw std::invalid_argument("geometry_project_batch: q must be (n, 2) or (n, 3)");
          }
          const int d = int(q.shape(1));
          const py::ssize_t n = q.shape(0);
          // One wire row: its kFields reals, and the row's slice of each
          // segmented field appended to an arena that the record addresses.
          std::vector<double> rec(EGG_B200_ENTITY_FIELDS, 0.0), arena;
          for (py::ssize_t i = 0; i < std::min<py::ssize_t>(records.size(), EGG_B200_ENTITY_FIELDS); ++i) {
              rec[size_t(i)] = records.data()[i];
          }
          int k = 0;
          std::vector<double> seg_at, seg_len;
          for (auto item : seg) {
              py::dict sd = item.cast<py::dict>();
              DArr data = DArr::ensure(sd["data"]);
              IArr off = IArr::ensure(sd["off"]);
              if (!data || !off || off.size() < 2 || off.data()[0] < 0 || off.data()[1] > data.size() ||
                  off.data()[0] > off.data()[1]) {
                  throw std::invalid_argument("geometry_project_batch: seg slot " + std::to_string(k) + " is malformed");
              }
              const double base = double(arena.size());
              if (tag == EGG_B200_TAG_BSPLINE && k < 3) { rec[size_t(6 + k)] = base; }
              if (tag == EGG_B200_TAG_COMPOSITE && k == 0) { rec[6] = base; }
              if (tag == EGG_B200_TAG_BSPLINESURF && k < 4) { rec[size_t(4 + k)] = base; }
              seg_at.push_back(base);
              seg_len.push_back(double(off.data()[1] - off.data()[0]));
              arena.insert(arena.end(), data.data() + off.data()[0], data.data() + off.data()[1]);
              ++k;
          }
          if (tag == EGG_B200_TAG_BSPLINESURF) {  // the UV trim through its header
              rec[9] = -1.0;
              if (seg_at.size() >= 6 && seg_len[5] >= 2) {
                  rec[9] = double(arena.size());
                  arena.push_back(seg_len[5]);
                  arena.push_back(seg_at[5]);
                  arena.push_back(seg_at[4]);
              }
          }
          const bool surf = d == 3 && (tag == EGG_B200_TAG_PLANE || tag == EGG_B200_TAG_SPHERE ||
                                       tag == EGG_B200_TAG_CYLINDER || tag == EGG_B200_TAG_BSPLINESURF);
          const int K = surf ? 2 : 1;
          py::array_t<double> feet({n, py::ssize_t(d)});
          py::array_t<double> basis({n, py::ssize_t(d), py::ssize_t(K)});
          check(egg_b200_entity_frame(d, tag, rec.data(), arena.empty() ? nullptr : arena.data(), int64_t(arena.size()),
                                      q.data(), int64_t(n), feet.mutable_data(), basis.mutable_data()));
          return std::make_tuple(feet, basis);
      },
      py::arg("q"), py::arg("tag"), py::arg("records"), py::arg("seg"),
      "Batched projection onto ONE entity in its wire (SoA) encoding, on the device. q is (n, d), d in {2, 3}; "
      "returns (feet(n, d), basis(n, d, tdim)): the projected points and the orthonormal tangent basis at each foot.");
    m.def(
      "energy_mindet",
      [](const DArr& X, const IArr& gc, const IArr& gn0, const IArr& gn1, const DArr& s0, const DArr& s1,
         const DArr& W) {
          const int P = int(gc.size());
          if (gn0.size() != P || gn1.size() != P || s0.size() != P || s1.size() != P || W.size() != 4 * P) {
              throw py::value_error("energy_mindet: inconsistent patch array sizes");
          }
          // every occurrence in role -1: the patch's energy and min det A, no gradient
          std::vector<int32_t> role(size_t(P), -1);
          std::vector<double> g(2), h(4), st(2);
          double e = 0, md = 0;
          check(egg_b200_patch_eval(EGG_B200_OBJ_SHAPE, 0.0, X.data(), int64_t(X.size() / 2), P, gc.data(), gn0.data(),
                                    gn1.data(), s0.data(), s1.data(), W.data(), role.data(), g.data(), h.data(), &e,
                                    &md, st.data()));
          return std::make_tuple(e, md);
      },
      py::arg("X"), py::arg("gc"), py::arg("gn0"), py::arg("gn1"), py::arg("s0"), py::arg("s1"), py::arg("W_inv"),
      "Patch energy and min det A only, on the GPU. Returns (energy, mindet).");
    m.def(
      "directional_eval",
      [](const py::array_t<double, py::array::c_style | py::array::forcecast>& X, const IArr& nodes, const IArr& kind,
         const py::array_t<double, py::array::c_style | py::array::forcecast>& ref, const DArr& weight, double eps) {
          if (X.ndim() != 2 || (X.shape(1) != 2 && X.shape(1) != 3)) {
              throw py::value_error("directional_eval: X must be (n_nodes, 2) or (n_nodes, 3)");
          }
          const int d = int(X.shape(1));
          const py::ssize_t n = weight.size();
          auto nb = nodes.request();
          if (nb.ndim != 2 || nb.shape[1] != 4 || nb.shape[0] != n || kind.size() != n || ref.ndim() != 2 ||
              ref.shape(0) != n || ref.shape(1) != d) {
              throw py::value_error("directional_eval: inconsistent sample-table shapes");
          }
          py::array_t<double> grad({X.shape(0), py::ssize_t(d)});
          double e = 0.0;
          check(egg_b200_directional_eval(d, X.data(), int64_t(X.shape(0)), int64_t(n), nodes.data(), kind.data(),
                                          ref.data(), weight.data(), eps, &e, grad.mutable_data()));
          return std::make_tuple(e, grad);
      },
      py::arg("X"), py::arg("nodes"), py::arg("kind"), py::arg("ref"), py::arg("weight"), py::arg("eps") = 1e-12,
      "Directional soft-energy total and gradient over a sample table, on the GPU. Returns (energy, grad (n_nodes, d)).");
    m.def(
      "wire_build",
      [](int dim, const IArr& shapes, const py::array_t<int64_t, py::array::c_style | py::array::forcecast>& ids,
         const py::array_t<uint8_t, py::array::c_style | py::array::forcecast>& moving, const py::object& stored,
         bool synth_interior, bool energy_arrays, const std::string& device) {
          if (dim != 2 && dim != 3) { throw py::value_error("wire_build: dim must be 2 or 3"); }
          if (shapes.size() % dim != 0) { throw py::value_error("wire_build: shapes length must be a multiple of dim"); }
          py::array_t<uint8_t, py::array::c_style | py::array::forcecast> st;
          if (!stored.is_none()) {
              st = py::array_t<uint8_t, py::array::c_style | py::array::forcecast>::ensure(stored);
              if (!st || st.size() != moving.size()) {
                  throw py::value_error("wire_build: stored must be a mask of num_nodes entries");
              }
          }
          egg_b200_wire_desc d {};
          d.dim = dim;
          d.num_blocks = int32_t(shapes.size() / dim);
          d.shapes = shapes.data();
          d.block_ids = ids.data();
          d.num_nodes = int64_t(moving.size());
          d.moving = moving.data();
          d.stored = stored.is_none() ? nullptr : st.data();
          d.synth_interior = synth_interior ? 1 : 0;
          d.energy_arrays = energy_arrays ? 1 : 0;
          d.device = device_of(device);
          int64_t total = 1;
          int64_t want = 0;
          for (int b = 0; b < d.num_blocks; ++b) {
              total = 1;
              for (int k = 0; k < dim; ++k) { total *= shapes.data()[b * dim + k]; }
              want += total;
          }
          if (int64_t(ids.size()) != want) { throw py::value_error("wire_build: block_ids length != sum of prod(shape)"); }
          egg_b200_wire* w = nullptr;
          int rc = EGG_B200_OK;
          {
              py::gil_scoped_release nogil;
              rc = egg_b200_wire_build(&d, &w);
          }
          check(rc);
          std::unique_ptr<egg_b200_wire, int (*)(egg_b200_wire*)> guard(w, egg_b200_wire_destroy);
          int64_t sz[3] = {0, 0, 0};
          check(egg_b200_wire_sizes(w, sz));
          const py::ssize_t nd = sz[0], nr = sz[1], ns = sz[2];
          py::dict out;
          egg_b200_wire_out o {};
          std::vector<std::pair<char*, size_t>> out_spans;
          auto iarr = [&](const char* key, py::ssize_t n) {
              py::array_t<int32_t> a(n);
              out[key] = a;
              out_spans.emplace_back(reinterpret_cast<char*>(a.mutable_data()), size_t(n) * sizeof(int32_t));
              return a.mutable_data();
          };
          auto darr = [&](const char* key, py::ssize_t n) {
              py::array_t<double> a(n);
              out[key] = a;
              out_spans.emplace_back(reinterpret_cast<char*>(a.mutable_data()), size_t(n) * sizeof(double));
              return a.mutable_data();
          };
          o.dof_idx = iarr("dof_idx", nd);
          o.P_of = iarr("P_of", nd);
          o.interior_block = iarr("interior_block", nd);
          {
              py::array_t<int32_t> a({nd, py::ssize_t(dim)});
              out["interior_logical"] = a;
              o.interior_logical = a.mutable_data();
          }
          o.role = iarr("role", nr);
          {
              py::array_t<int64_t> a(nr);
              out["sid"] = a;
              o.sid = a.mutable_data();
          }
          o.gc = iarr("gc", nr);
          const char* gnk[3] = {"gn0", "gn1", "gn2"};
          const char* sk[3] = {"s0", "s1", "s2"};
          const char* es_gnk[3] = {"es_gn0", "es_gn1", "es_gn2"};
          const char* es_sk[3] = {"es_s0", "es_s1", "es_s2"};
          for (int k = 0; k < dim; ++k) {
              o.gn[k] = iarr(gnk[k], nr);
              o.s[k] = darr(sk[k], nr);
          }
          if (energy_arrays) {
              o.es_gc = iarr("es_gc", ns);
              for (int k = 0; k < dim; ++k) {
                  o.es_gn[k] = iarr(es_gnk[k], ns);
                  o.es_s[k] = darr(es_sk[k], ns);
              }
          }
          out["num_samples"] = ns;
          {
              py::gil_scoped_release nogil;
              // Fresh arrays fault in their pages on first touch; touch them
              // on several threads first, so the copies land in resident pages.
              prefault(out_spans);
              rc = egg_b200_wire_download(w, &o);
          }
          check(rc);
          return out;
      },
      py::arg("dim"), py::arg("shapes"), py::arg("block_ids"), py::arg("moving"), py::arg("stored") = py::none(),
      py::arg("synth_interior") = true, py::arg("energy_arrays") = true, py::arg("device") = "auto",
      "Device-side build of the sweep-context wire's index arrays (the array work of build_flat_context): "
      "returns a dict of the group's dof_idx, P_of, interior_block, interior_logical, role, sid, gc, gn*, s* and, "
      "with energy_arrays, the energy stencil's es_gc, es_gn*, es_s*, plus num_samples.");
}
