// gfb_files.cpp -- raw (.gfr) and HDF5 (.h5) dataset files for the
// file-level driver (see gfb_files.h).
#include "gfb_files.h"

#include <cerrno>
#include <cstdio>
#include <cstring>
#include <type_traits>

#ifndef GFB_HAVE_HDF5
#define GFB_HAVE_HDF5 0
#endif
#if GFB_HAVE_HDF5
#include <hdf5.h>
#endif

namespace gfb {
namespace files {

namespace {

constexpr char kMagic[8] = {'G', 'F', 'B', 'R', 'A', 'W', '0', '1'};

size_t type_size(Type t) {
    switch (t) {
        case Type::F64: case Type::I64: return 8;
        case Type::F32: case Type::I32: return 4;
        default: return 1;
    }
}

bool ends_with(const std::string& s, const char* suffix) {
    const size_t n = std::strlen(suffix);
    return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

std::string attr_key(const std::string& obj, const std::string& name) {
    return (obj.empty() ? std::string("/") : obj) + "@" + name;
}

// ------------------------------------------------------------------ raw read

struct RawEntry {
    Type type;
    std::vector<uint64_t> dims;
    uint64_t offset = 0, bytes = 0;
};

class RawReader : public Reader {
public:
    ~RawReader() override {
        if (f_) std::fclose(f_);
    }

    bool open(const std::string& path, std::string& err) {
        f_ = std::fopen(path.c_str(), "rb");
        if (!f_) {
            err = "cannot open " + path + ": " + std::strerror(errno);
            return false;
        }
        char magic[8];
        uint32_t n = 0;
        if (std::fread(magic, 1, 8, f_) != 8 || std::memcmp(magic, kMagic, 8) != 0 || !get(&n, 4)) {
            err = path + " is not a GFBRAW01 container";
            return false;
        }
        for (uint32_t i = 0; i < n; ++i) {
            uint16_t len = 0;
            uint8_t type = 0, ndim = 0;
            if (!get(&len, 2)) return bad(path, err);
            std::string name(len, '\0');
            if (len && !get(&name[0], len)) return bad(path, err);
            if (!get(&type, 1) || !get(&ndim, 1) || type < 1 || type > 6 || ndim > 8) return bad(path, err);
            RawEntry e;
            e.type = static_cast<Type>(type);
            e.dims.resize(ndim);
            for (auto& d : e.dims)
                if (!get(&d, 8)) return bad(path, err);
            if (!get(&e.offset, 8) || !get(&e.bytes, 8)) return bad(path, err);
            uint64_t count = 1;
            for (auto d : e.dims) count *= d;
            if (e.type != Type::STR && count * type_size(e.type) != e.bytes) return bad(path, err);
            entries_[name] = std::move(e);
        }
        path_ = path;
        return true;
    }

    bool has_dataset(const std::string& path) const override {
        return path.find('@') == std::string::npos && entries_.count(path) > 0;
    }
    bool has_group(const std::string& path) const override {
        const std::string a = path + "/", b = path + "@";
        for (const auto& kv : entries_)
            if (kv.first.compare(0, a.size(), a) == 0 || kv.first.compare(0, b.size(), b) == 0) return true;
        return false;
    }
    std::vector<uint64_t> dims(const std::string& path) const override {
        auto it = entries_.find(path);
        return it == entries_.end() ? std::vector<uint64_t>{} : it->second.dims;
    }
    bool read_f64(const std::string& p, std::vector<double>& out) const override { return read_num(p, out); }
    bool read_i64(const std::string& p, std::vector<int64_t>& out) const override { return read_num(p, out); }
    bool read_i32(const std::string& p, std::vector<int32_t>& out) const override { return read_num(p, out); }

    bool attr_f64(const std::string& obj, const std::string& name, double& out) const override {
        std::vector<double> v;
        if (!read_num(attr_key(obj, name), v) || v.size() != 1) return false;
        out = v[0];
        return true;
    }
    bool attr_i32(const std::string& obj, const std::string& name, int& out) const override {
        std::vector<int64_t> v;
        if (!read_num(attr_key(obj, name), v) || v.size() != 1) return false;
        out = (int)v[0];
        return true;
    }
    bool attr_str(const std::string& obj, const std::string& name, std::string& out) const override {
        auto it = entries_.find(attr_key(obj, name));
        if (it == entries_.end() || it->second.type != Type::STR) return false;
        out.assign(it->second.bytes, '\0');
        return read_bytes(it->second, &out[0]);
    }

private:
    FILE* f_ = nullptr;
    std::string path_;
    std::map<std::string, RawEntry> entries_;

    bool get(void* p, size_t n) { return std::fread(p, 1, n, f_) == n; }
    static bool bad(const std::string& path, std::string& err) {
        err = path + ": truncated or malformed GFBRAW01 header";
        return false;
    }
    bool read_bytes(const RawEntry& e, void* dst) const {
        if (e.bytes == 0) return true;
        if (std::fseek(f_, (long)e.offset, SEEK_SET) != 0) return false;
        return std::fread(dst, 1, e.bytes, f_) == e.bytes;
    }
    template <typename T>
    bool read_num(const std::string& path, std::vector<T>& out) const {
        auto it = entries_.find(path);
        if (it == entries_.end() || it->second.type == Type::STR) return false;
        const RawEntry& e = it->second;
        const size_t n = e.bytes / type_size(e.type);
        out.resize(n);
        switch (e.type) {
            case Type::F64: return convert<double>(e, out);
            case Type::F32: return convert<float>(e, out);
            case Type::I64: return convert<int64_t>(e, out);
            case Type::I32: return convert<int32_t>(e, out);
            case Type::U8: return convert<uint8_t>(e, out);
            default: return false;
        }
    }
    template <typename S, typename T>
    bool convert(const RawEntry& e, std::vector<T>& out) const {
        if (std::is_same<S, T>::value) return read_bytes(e, out.data());
        std::vector<S> tmp(out.size());
        if (!read_bytes(e, tmp.data())) return false;
        for (size_t i = 0; i < tmp.size(); ++i) out[i] = static_cast<T>(tmp[i]);
        return true;
    }
};

// ----------------------------------------------------------------- raw write

class RawWriter : public Writer {
public:
    explicit RawWriter(std::string path) : path_(std::move(path)) {}

    void attr_str(const std::string& obj, const std::string& name, const std::string& v) override {
        add_owned(attr_key(obj, name), Type::STR, {v.size()}, v.data(), v.size());
    }
    void attr_i32(const std::string& obj, const std::string& name, int v) override {
        const int32_t x = v;
        add_owned(attr_key(obj, name), Type::I32, {}, &x, 4);
    }
    void attr_f64(const std::string& obj, const std::string& name, double v) override {
        add_owned(attr_key(obj, name), Type::F64, {}, &v, 8);
    }
    void attr_bool(const std::string& obj, const std::string& name, bool v) override {
        const uint8_t x = v ? 1 : 0;
        add_owned(attr_key(obj, name), Type::U8, {}, &x, 1);
    }
    // Non-owning: data must stay valid until close().
    void dataset(const std::string& path, Type type, const std::vector<uint64_t>& dims, const void* data,
                 bool) override {
        uint64_t n = 1;
        for (auto d : dims) n *= d;
        Item it;
        it.name = path;
        it.type = type;
        it.dims = dims;
        it.data = data;
        it.bytes = n * type_size(type);
        items_.push_back(std::move(it));
    }

    bool close(std::string& err) override {
        FILE* f = std::fopen(path_.c_str(), "wb");
        if (!f) {
            err = "cannot create " + path_ + ": " + std::strerror(errno);
            return false;
        }
        uint64_t header = 8 + 4;
        for (const auto& it : items_) header += 2 + it.name.size() + 2 + 8 * it.dims.size() + 16;
        uint64_t off = (header + 63) / 64 * 64;
        std::vector<uint64_t> offs;
        for (const auto& it : items_) {
            offs.push_back(off);
            off = (off + it.bytes + 63) / 64 * 64;
        }
        bool ok = std::fwrite(kMagic, 1, 8, f) == 8;
        const uint32_t n = (uint32_t)items_.size();
        ok = ok && std::fwrite(&n, 4, 1, f) == 1;
        for (size_t i = 0; ok && i < items_.size(); ++i) {
            const auto& it = items_[i];
            const uint16_t len = (uint16_t)it.name.size();
            const uint8_t type = (uint8_t)it.type, ndim = (uint8_t)it.dims.size();
            ok = std::fwrite(&len, 2, 1, f) == 1 && std::fwrite(it.name.data(), 1, len, f) == len &&
                 std::fwrite(&type, 1, 1, f) == 1 && std::fwrite(&ndim, 1, 1, f) == 1;
            for (auto d : it.dims) ok = ok && std::fwrite(&d, 8, 1, f) == 1;
            ok = ok && std::fwrite(&offs[i], 8, 1, f) == 1 && std::fwrite(&it.bytes, 8, 1, f) == 1;
        }
        uint64_t pos = header;
        static const char zeros[64] = {};
        for (size_t i = 0; ok && i < items_.size(); ++i) {
            if (offs[i] > pos) ok = std::fwrite(zeros, 1, offs[i] - pos, f) == offs[i] - pos;
            const void* src = items_[i].owned.empty() ? items_[i].data : items_[i].owned.data();
            if (ok && items_[i].bytes) ok = std::fwrite(src, 1, items_[i].bytes, f) == items_[i].bytes;
            pos = offs[i] + items_[i].bytes;
        }
        if (std::fclose(f) != 0) ok = false;
        if (!ok) err = "write failed: " + path_;
        return ok;
    }

private:
    struct Item {
        std::string name;
        Type type;
        std::vector<uint64_t> dims;
        const void* data = nullptr;
        std::vector<char> owned;
        uint64_t bytes = 0;
    };
    std::string path_;
    std::vector<Item> items_;

    void add_owned(const std::string& name, Type type, std::vector<uint64_t> dims, const void* p, size_t n) {
        Item it;
        it.name = name;
        it.type = type;
        it.dims = std::move(dims);
        it.owned.assign(static_cast<const char*>(p), static_cast<const char*>(p) + n);
        it.bytes = n;
        items_.push_back(std::move(it));
    }
};

#if GFB_HAVE_HDF5
// ------------------------------------------------------------------ HDF5

hid_t native(Type t) {
    switch (t) {
        case Type::F64: return H5T_NATIVE_DOUBLE;
        case Type::F32: return H5T_NATIVE_FLOAT;
        case Type::I64: return H5T_NATIVE_INT64;
        case Type::I32: return H5T_NATIVE_INT32;
        default: return H5T_NATIVE_UINT8;
    }
}

class H5Reader : public Reader {
public:
    ~H5Reader() override {
        if (f_ >= 0) H5Fclose(f_);
    }
    bool open(const std::string& path, std::string& err) {
        H5E_BEGIN_TRY { f_ = H5Fopen(path.c_str(), H5F_ACC_RDONLY, H5P_DEFAULT); }
        H5E_END_TRY;
        if (f_ < 0) err = "H5Fopen failed: " + path;
        return f_ >= 0;
    }
    bool has_dataset(const std::string& path) const override {
        htri_t e;
        H5E_BEGIN_TRY { e = H5Lexists(f_, path.c_str(), H5P_DEFAULT); }
        H5E_END_TRY;
        if (e <= 0) return false;
        H5O_info2_t info;
        if (H5Oget_info_by_name3(f_, path.c_str(), &info, H5O_INFO_BASIC, H5P_DEFAULT) < 0) return false;
        return info.type == H5O_TYPE_DATASET;
    }
    bool has_group(const std::string& path) const override {
        hid_t g;
        H5E_BEGIN_TRY { g = H5Gopen2(f_, path.c_str(), H5P_DEFAULT); }
        H5E_END_TRY;
        if (g < 0) return false;
        H5Gclose(g);
        return true;
    }
    std::vector<uint64_t> dims(const std::string& path) const override {
        std::vector<uint64_t> out;
        if (!has_dataset(path)) return out;
        hid_t d = H5Dopen2(f_, path.c_str(), H5P_DEFAULT);
        hid_t s = H5Dget_space(d);
        const int nd = H5Sget_simple_extent_ndims(s);
        hsize_t dd[16];
        if (nd > 0 && nd <= 16) {
            H5Sget_simple_extent_dims(s, dd, nullptr);
            out.assign(dd, dd + nd);
        }
        H5Sclose(s);
        H5Dclose(d);
        return out;
    }
    bool read_f64(const std::string& p, std::vector<double>& o) const override { return rd(p, o, H5T_NATIVE_DOUBLE); }
    bool read_i64(const std::string& p, std::vector<int64_t>& o) const override { return rd(p, o, H5T_NATIVE_INT64); }
    bool read_i32(const std::string& p, std::vector<int32_t>& o) const override { return rd(p, o, H5T_NATIVE_INT32); }
    bool attr_f64(const std::string& obj, const std::string& name, double& out) const override {
        return attr(obj, name, H5T_NATIVE_DOUBLE, &out);
    }
    bool attr_i32(const std::string& obj, const std::string& name, int& out) const override {
        return attr(obj, name, H5T_NATIVE_INT, &out);
    }
    bool attr_str(const std::string& obj, const std::string& name, std::string& out) const override {
        hid_t a = open_attr(obj, name);
        if (a < 0) return false;
        hid_t t = H5Aget_type(a);
        bool ok = false;
        if (H5Tis_variable_str(t) > 0) {
            char* v = nullptr;
            ok = H5Aread(a, t, &v) >= 0;
            if (ok) out = v ? v : "";
            if (v) H5free_memory(v);
        } else {
            std::vector<char> buf(H5Tget_size(t) + 1, '\0');
            ok = H5Aread(a, t, buf.data()) >= 0;
            if (ok) out = buf.data();
        }
        H5Tclose(t);
        H5Aclose(a);
        return ok;
    }

private:
    hid_t f_ = -1;
    template <typename T>
    bool rd(const std::string& path, std::vector<T>& out, hid_t mem) const {
        if (!has_dataset(path)) return false;
        uint64_t n = 1;
        for (auto d : dims(path)) n *= d;
        out.resize(n);
        hid_t d = H5Dopen2(f_, path.c_str(), H5P_DEFAULT);
        const bool ok = d >= 0 && (n == 0 || H5Dread(d, mem, H5S_ALL, H5S_ALL, H5P_DEFAULT, out.data()) >= 0);
        if (d >= 0) H5Dclose(d);
        return ok;
    }
    hid_t open_attr(const std::string& obj, const std::string& name) const {
        hid_t a;
        H5E_BEGIN_TRY {
            a = H5Aexists_by_name(f_, obj.c_str(), name.c_str(), H5P_DEFAULT) > 0
                    ? H5Aopen_by_name(f_, obj.c_str(), name.c_str(), H5P_DEFAULT, H5P_DEFAULT)
                    : -1;
        }
        H5E_END_TRY;
        return a;
    }
    bool attr(const std::string& obj, const std::string& name, hid_t mem, void* out) const {
        hid_t a = open_attr(obj, name);
        if (a < 0) return false;
        const bool ok = H5Aread(a, mem, out) >= 0;
        H5Aclose(a);
        return ok;
    }
};

class H5Writer : public Writer {
public:
    ~H5Writer() override {
        if (f_ >= 0) H5Fclose(f_);
    }
    bool create(const std::string& path, std::string& err) {
        f_ = H5Fcreate(path.c_str(), H5F_ACC_TRUNC, H5P_DEFAULT, H5P_DEFAULT);
        if (f_ < 0) err = "H5Fcreate failed: " + path;
        return f_ >= 0;
    }
    void attr_str(const std::string& obj, const std::string& name, const std::string& v) override {
        hid_t t = H5Tcopy(H5T_C_S1);
        H5Tset_size(t, v.size() ? v.size() : 1);
        put_attr(obj, name, t, v.c_str());
        H5Tclose(t);
    }
    void attr_i32(const std::string& obj, const std::string& name, int v) override {
        put_attr(obj, name, H5T_NATIVE_INT, &v);
    }
    void attr_f64(const std::string& obj, const std::string& name, double v) override {
        put_attr(obj, name, H5T_NATIVE_DOUBLE, &v);
    }
    void attr_bool(const std::string& obj, const std::string& name, bool v) override {
        const hbool_t b = v ? 1 : 0;
        put_attr(obj, name, H5T_NATIVE_HBOOL, &b);
    }
    void dataset(const std::string& path, Type type, const std::vector<uint64_t>& dims, const void* data,
                 bool chunk) override {
        std::vector<hsize_t> d(dims.begin(), dims.end());
        hid_t s = H5Screate_simple((int)d.size(), d.data(), nullptr);
        hid_t pl = H5Pcreate(H5P_DATASET_CREATE);
        if (chunk) H5Pset_chunk(pl, (int)d.size(), d.data());
        hid_t ds = H5Dcreate2(f_, path.c_str(), native(type), s, H5P_DEFAULT, pl, H5P_DEFAULT);
        if (ds < 0 || H5Dwrite(ds, native(type), H5S_ALL, H5S_ALL, H5P_DEFAULT, data) < 0) failed_ = true;
        if (ds >= 0) H5Dclose(ds);
        H5Pclose(pl);
        H5Sclose(s);
    }
    bool close(std::string& err) override {
        const bool ok = !failed_ && f_ >= 0 && H5Fclose(f_) >= 0;
        f_ = -1;
        if (!ok) err = "HDF5 write failed";
        return ok;
    }

private:
    hid_t f_ = -1;
    bool failed_ = false;
    void put_attr(const std::string& obj, const std::string& name, hid_t type, const void* v) {
        hid_t s = H5Screate(H5S_SCALAR);
        hid_t a = H5Acreate_by_name(f_, obj.c_str(), name.c_str(), type, s, H5P_DEFAULT, H5P_DEFAULT, H5P_DEFAULT);
        if (a < 0 || H5Awrite(a, type, v) < 0) failed_ = true;
        if (a >= 0) H5Aclose(a);
        H5Sclose(s);
    }
};
#endif

}  // namespace

bool have_hdf5() { return GFB_HAVE_HDF5 != 0; }

std::unique_ptr<Reader> open_reader(const std::string& path, std::string& err) {
    if (ends_with(path, ".h5")) {
#if GFB_HAVE_HDF5
        auto r = std::make_unique<H5Reader>();
        if (!r->open(path, err)) return nullptr;
        return r;
#else
        err = "cannot read " + path + ": this build has no HDF5 (use the .gfr container)";
        return nullptr;
#endif
    }
    auto r = std::make_unique<RawReader>();
    if (!r->open(path, err)) return nullptr;
    return r;
}

std::unique_ptr<Writer> create_writer(const std::string& path, std::string& err) {
    if (ends_with(path, ".h5")) {
#if GFB_HAVE_HDF5
        auto w = std::make_unique<H5Writer>();
        if (!w->create(path, err)) return nullptr;
        return w;
#else
        err = "cannot write " + path + ": this build has no HDF5 (use the .gfr container)";
        return nullptr;
#endif
    }
    // check now that the file can be created, as H5Fcreate does
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        err = "cannot create " + path + ": " + std::strerror(errno);
        return nullptr;
    }
    std::fclose(f);
    return std::make_unique<RawWriter>(path);
}

}  // namespace files
}  // namespace gfb
