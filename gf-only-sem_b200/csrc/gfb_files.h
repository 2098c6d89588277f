// gfb_files.h -- dataset files of the file-level driver (gfb_run_forward).
//
// The reference's driver reads and writes HDF5 files through a handful of
// calls: datasets by path ("/field/cell/dxi_dx"), attributes of a group or
// of the file ("/simulation" solver_dt), group existence, and one writer per
// output file (forward/share/src/io.cpp, record.cpp, restart.cpp).  This
// header gives the driver that model over two containers:
//
//  * HDF5 (.h5), the reference's own files, when the library is built with
//    GFB_HAVE_HDF5 (libhdf5 headers and library present);
//  * a raw container (.gfr) with the same dataset and attribute names, for
//    hosts without HDF5.  Layout, little-endian:
//      "GFBRAW01"  u32 n_entries  then per entry:
//        u16 name_len, name (dataset path, or "<object path>@<attribute>"),
//        u8 type (1 f64, 2 f32, 3 i64, 4 i32, 5 u8, 6 string), u8 ndim,
//        u64 dims[ndim], u64 offset (from the file start), u64 bytes
//      then the data blocks, each starting on a 64-byte boundary.
//    A group exists when an entry's name lies under it.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace gfb {
namespace files {

enum class Type : uint8_t { F64 = 1, F32 = 2, I64 = 3, I32 = 4, U8 = 5, STR = 6 };

// Read side.  Numeric reads convert from the stored type to T.
class Reader {
public:
    virtual ~Reader() = default;
    virtual bool has_dataset(const std::string& path) const = 0;
    virtual bool has_group(const std::string& path) const = 0;
    // dims of a dataset (empty when absent)
    virtual std::vector<uint64_t> dims(const std::string& path) const = 0;
    virtual bool read_f64(const std::string& path, std::vector<double>& out) const = 0;
    virtual bool read_i64(const std::string& path, std::vector<int64_t>& out) const = 0;
    virtual bool read_i32(const std::string& path, std::vector<int32_t>& out) const = 0;
    // attributes of the object at `obj` ("/" for the file)
    virtual bool attr_f64(const std::string& obj, const std::string& name, double& out) const = 0;
    virtual bool attr_i32(const std::string& obj, const std::string& name, int& out) const = 0;
    virtual bool attr_str(const std::string& obj, const std::string& name, std::string& out) const = 0;
};

// Write side: one output file, written when close() is called (raw) or as
// the calls come (HDF5).  `chunk` asks for one chunk of the whole dataset
// (the record datasets of record.cpp:103-142).
class Writer {
public:
    virtual ~Writer() = default;
    virtual void attr_str(const std::string& obj, const std::string& name, const std::string& v) = 0;
    virtual void attr_i32(const std::string& obj, const std::string& name, int v) = 0;
    virtual void attr_f64(const std::string& obj, const std::string& name, double v) = 0;
    virtual void attr_bool(const std::string& obj, const std::string& name, bool v) = 0;
    virtual void dataset(const std::string& path, Type type, const std::vector<uint64_t>& dims, const void* data,
                         bool chunk = false) = 0;
    // false with err set on failure; the file is complete after it
    virtual bool close(std::string& err) = 0;
};

// Open an input file; the container follows the extension (.gfr raw, .h5
// HDF5).  Returns null with err set on failure.
std::unique_ptr<Reader> open_reader(const std::string& path, std::string& err);
// Create (truncate) an output file of the container of its extension.
std::unique_ptr<Writer> create_writer(const std::string& path, std::string& err);

// Whether this build reads and writes HDF5 files.
bool have_hdf5();

}  // namespace files
}  // namespace gfb
