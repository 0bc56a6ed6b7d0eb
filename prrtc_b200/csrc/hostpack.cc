// hostpack.cc -- native host packer for uneven per-problem worlds (CPython
// extension module prrtc_b200._hostpack).
//
// prrtc_plan_batch packs the world / self tables of B collision_context dicts
// into padded [B, max_n, feat] tables plus per-problem row counts (the layout
// of prrtc.py:1009-1067).  Done in Python that is a few thousand dict lookups
// and array checks per call, which dominates the host side of a batch call.
// This module walks the contexts once to size the tables (scan) and once to
// write them straight into the caller's pinned staging buffer (fill).  Tables
// are read through the buffer protocol: C-contiguous 2-D arrays of 4-byte
// float32 ('f') or int32 ('i') items.  Anything else raises TypeError and the
// caller uses its Python packer.  numpy arrays are read through the numpy C
// API (data pointer, shape and flags straight from the array object): the
// buffer protocol costs a few hundred nanoseconds per array, which over 512
// contexts x 5 tables x 2 passes was most of the host time of a batch call.
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#define NPY_NO_DEPRECATED_API NPY_1_7_API_VERSION
#include <numpy/arrayobject.h>

#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct Spec {
    const char* key;
    Py_ssize_t feat;
    char kind;  // 'f' float32, 'i' int32
};

bool format_ok(const Py_buffer& b, char kind) {
    if (b.itemsize != 4 || b.format == nullptr) return false;
    const char* f = b.format;
    if (*f == '<' || *f == '=' || *f == '@') ++f;
    if (kind == 'f') return f[0] == 'f' && f[1] == 0;
    return (f[0] == 'i' || f[0] == 'l') && f[1] == 0 && b.itemsize == 4;
}

// One table view: the object (borrowed), its data, its row count (and the
// buffer held for a non-numpy object).
struct Table {
    PyObject* obj = nullptr;
    const void* data = nullptr;
    Py_ssize_t rows = 0, bytes = 0;
    Py_buffer buf{};
    bool held = false;
};

struct Tables {
    std::vector<Table> t;
    ~Tables() {
        for (auto& x : t)
            if (x.held) PyBuffer_Release(&x.buf);
    }
};

bool parse_specs(PyObject* specs, std::vector<Spec>& out) {
    PyObject* seq = PySequence_Fast(specs, "specs must be a sequence of (key, feat, kind)");
    if (!seq) return false;
    const Py_ssize_t n = PySequence_Fast_GET_SIZE(seq);
    for (Py_ssize_t i = 0; i < n; ++i) {
        PyObject* it = PySequence_Fast_GET_ITEM(seq, i);
        const char* key;
        Py_ssize_t feat;
        int kind;
        if (!PyArg_ParseTuple(it, "snC", &key, &feat, &kind)) {
            Py_DECREF(seq);
            return false;
        }
        out.push_back({key, feat, (char)kind});
    }
    Py_DECREF(seq);
    return true;
}

// Fill tabs[i] with key `s` of context i (absent / None context = no table).
bool gather(PyObject* ctx_seq, const Spec& s, Tables& tabs) {
    const Py_ssize_t B = PySequence_Fast_GET_SIZE(ctx_seq);
    tabs.t.assign((size_t)B, Table{});
    PyObject* key = PyUnicode_InternFromString(s.key);  // one hashed key object for every lookup
    if (!key) return false;
    const int npy_type = s.kind == 'f' ? NPY_FLOAT32 : NPY_INT32;
    bool ok = true;
    for (Py_ssize_t i = 0; i < B && ok; ++i) {
        PyObject* c = PySequence_Fast_GET_ITEM(ctx_seq, i);
        if (c == Py_None) continue;
        if (!PyDict_Check(c)) {
            PyErr_SetString(PyExc_TypeError, "collision_context entries must be dicts");
            ok = false;
            break;
        }
        PyObject* x = PyDict_GetItemWithError(c, key);  // borrowed
        if (x == nullptr) {
            if (PyErr_Occurred()) ok = false;
            continue;
        }
        if (x == Py_None) continue;
        Table& t = tabs.t[(size_t)i];
        t.obj = x;
        if (PyArray_Check(x)) {
            PyArrayObject* a = reinterpret_cast<PyArrayObject*>(x);
            if (PyArray_NDIM(a) != 2 || PyArray_DIM(a, 1) != s.feat || PyArray_TYPE(a) != npy_type ||
                PyArray_ITEMSIZE(a) != 4 || !PyArray_ISCARRAY_RO(a)) {
                PyErr_Format(PyExc_TypeError, "collision_context[%zd]['%s'] is not a C-contiguous (N, %zd) %s array",
                             i, s.key, s.feat, s.kind == 'f' ? "float32" : "int32");
                ok = false;
                break;
            }
            t.data = PyArray_DATA(a);
            t.rows = PyArray_DIM(a, 0);
            t.bytes = t.rows * s.feat * 4;
            continue;
        }
        if (PyObject_GetBuffer(x, &t.buf, PyBUF_C_CONTIGUOUS | PyBUF_FORMAT) != 0) {
            PyErr_Clear();
            PyErr_Format(PyExc_TypeError, "collision_context[%zd]['%s'] has no contiguous buffer", i, s.key);
            ok = false;
            break;
        }
        t.held = true;
        if (t.buf.ndim != 2 || t.buf.shape[1] != s.feat || !format_ok(t.buf, s.kind)) {
            PyErr_Format(PyExc_TypeError, "collision_context[%zd]['%s'] is not a (N, %zd) %s array", i, s.key, s.feat,
                         s.kind == 'f' ? "float32" : "int32");
            ok = false;
            break;
        }
        t.data = t.buf.buf;
        t.rows = t.buf.shape[0];
        t.bytes = t.buf.len;
    }
    Py_DECREF(key);
    return ok;
}

// Every context holds the same table (same object or equal bytes; an empty
// table matches any of the same shape), the first context included.
bool shared(const Tables& tabs) {
    if (tabs.t.empty() || tabs.t[0].obj == nullptr) return false;
    const Table& a = tabs.t[0];
    for (size_t i = 1; i < tabs.t.size(); ++i) {
        const Table& x = tabs.t[i];
        if (x.obj == nullptr) return false;
        if (x.obj == a.obj) continue;
        if (x.rows != a.rows) return false;
        if (x.rows == 0) continue;
        if (std::memcmp(x.data, a.data, (size_t)a.bytes) != 0) return false;
    }
    return true;
}

// scan(contexts, specs) -> tuple per spec of (shared, max_rows, counts: bytes of int32[B])
PyObject* scan(PyObject*, PyObject* args) {
    PyObject *contexts, *specs;
    if (!PyArg_ParseTuple(args, "OO", &contexts, &specs)) return nullptr;
    std::vector<Spec> sp;
    if (!parse_specs(specs, sp)) return nullptr;
    PyObject* seq = PySequence_Fast(contexts, "contexts must be a sequence");
    if (!seq) return nullptr;
    const Py_ssize_t B = PySequence_Fast_GET_SIZE(seq);
    PyObject* out = PyTuple_New((Py_ssize_t)sp.size());
    for (size_t k = 0; k < sp.size() && out; ++k) {
        Tables tabs;
        if (!gather(seq, sp[k], tabs)) {
            Py_CLEAR(out);
            break;
        }
        std::vector<int32_t> counts((size_t)B);
        Py_ssize_t mx = 0;
        for (Py_ssize_t i = 0; i < B; ++i) {
            const Py_ssize_t r = tabs.t[(size_t)i].rows;
            if (r > INT32_MAX) {
                PyErr_SetString(PyExc_ValueError, "table too large");
                Py_CLEAR(out);
                break;
            }
            counts[(size_t)i] = (int32_t)r;
            if (r > mx) mx = r;
        }
        if (!out) break;
        PyObject* item = Py_BuildValue("(Nny#)", PyBool_FromLong(shared(tabs)), mx,
                                       reinterpret_cast<const char*>(counts.data()), (Py_ssize_t)(B * 4));
        if (!item) {
            Py_CLEAR(out);
            break;
        }
        PyTuple_SET_ITEM(out, (Py_ssize_t)k, item);
    }
    Py_DECREF(seq);
    return out;
}

// fill(contexts, specs, layout, out): layout per spec is (shared, max_rows,
// table_offset, counts_offset); a shared spec copies context 0's table, the
// others write the rows of a [B, max_rows, feat] table and int32[B] counts
// (counts_offset < 0: no counts).  Rows past a problem's count are left as
// they were: the planner reads only counted rows.  Offsets are bytes into
// the writable `out`.
PyObject* fill(PyObject*, PyObject* args) {
    PyObject *contexts, *specs, *layout, *outobj;
    if (!PyArg_ParseTuple(args, "OOOO", &contexts, &specs, &layout, &outobj)) return nullptr;
    std::vector<Spec> sp;
    if (!parse_specs(specs, sp)) return nullptr;
    Py_buffer ob;
    if (PyObject_GetBuffer(outobj, &ob, PyBUF_WRITABLE | PyBUF_C_CONTIGUOUS) != 0) return nullptr;
    PyObject* seq = PySequence_Fast(contexts, "contexts must be a sequence");
    PyObject* lay = seq ? PySequence_Fast(layout, "layout must be a sequence") : nullptr;
    bool ok = seq && lay && PySequence_Fast_GET_SIZE(lay) == (Py_ssize_t)sp.size();
    if (seq && lay && !ok) PyErr_SetString(PyExc_ValueError, "layout and specs differ in length");
    unsigned char* base = static_cast<unsigned char*>(ob.buf);
    const Py_ssize_t B = ok ? PySequence_Fast_GET_SIZE(seq) : 0;
    for (size_t k = 0; ok && k < sp.size(); ++k) {
        int is_shared;
        Py_ssize_t mx, toff, coff;
        if (!PyArg_ParseTuple(PySequence_Fast_GET_ITEM(lay, (Py_ssize_t)k), "pnnn", &is_shared, &mx, &toff, &coff)) {
            ok = false;
            break;
        }
        Tables tabs;
        if (!gather(seq, sp[k], tabs)) {
            ok = false;
            break;
        }
        const Py_ssize_t row_bytes = sp[k].feat * 4;
        if (is_shared) {
            const Table& a = tabs.t.empty() ? Table{} : tabs.t[0];
            const Py_ssize_t n = a.rows * row_bytes;
            if (a.rows != mx) {  // the table changed since scan(): its reserved region no longer fits
                PyErr_SetString(PyExc_ValueError, "a shared table's row count differs from the layout's");
                ok = false;
                break;
            }
            if (toff < 0 || toff + n > ob.len) {
                PyErr_SetString(PyExc_ValueError, "staging buffer too small");
                ok = false;
                break;
            }
            if (n) std::memcpy(base + toff, a.data, (size_t)n);
            continue;
        }
        const Py_ssize_t tb = B * mx * row_bytes;
        if (toff < 0 || toff + tb > ob.len || (coff >= 0 && coff + B * 4 > ob.len)) {
            PyErr_SetString(PyExc_ValueError, "staging buffer too small");
            ok = false;
            break;
        }
        for (Py_ssize_t i = 0; i < B; ++i) {
            const Table& t = tabs.t[(size_t)i];
            if (t.rows > mx) {
                PyErr_SetString(PyExc_ValueError, "a table has more rows than the layout's max_rows");
                ok = false;
                break;
            }
            if (t.rows) std::memcpy(base + toff + i * mx * row_bytes, t.data, (size_t)(t.rows * row_bytes));
            if (coff >= 0) {
                const int32_t r = (int32_t)t.rows;
                std::memcpy(base + coff + i * 4, &r, 4);
            }
        }
    }
    Py_XDECREF(lay);
    Py_XDECREF(seq);
    PyBuffer_Release(&ob);
    if (!ok) return nullptr;
    Py_RETURN_NONE;
}

PyMethodDef methods[] = {
    {"scan", scan, METH_VARARGS, "scan(contexts, specs) -> per spec (shared, max_rows, counts bytes)"},
    {"fill", fill, METH_VARARGS, "fill(contexts, specs, layout, out) -> None"},
    {nullptr, nullptr, 0, nullptr},
};

PyModuleDef module = {PyModuleDef_HEAD_INIT, "_hostpack", "Native host packer for per-problem worlds.", -1, methods};

}  // namespace

PyMODINIT_FUNC PyInit__hostpack(void) {
    import_array();  // numpy C API table (returns NULL with an ImportError set on failure)
    return PyModule_Create(&module);
}
