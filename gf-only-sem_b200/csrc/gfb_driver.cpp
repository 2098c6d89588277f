// gfb_driver.cpp -- file-level driver of the time loop: what
// `gf_solver_elastic_cuda --direction {x,y,z} [--resume]` runs
// (forward/share/src/solver.cpp:73-739 run_forward), over the library's C ABI.
//
// All paths are relative to the working directory, as the reference's:
//   in:   config.<ext>, partitions/partition_{r}.<ext> for r = 0, 1, ...
//         (all partitions merged onto the one GPU, io.cpp:319-450)
//   out:  wavefields/{dir}/record_0_{step}.<ext> per snapshot (record.cpp:175-257)
//         wavefields/{dir}/restart_0.<ext> (restart.cpp:87-152)
//         log/forward_{dir}_0.log (logger.hpp:23-30)
// <ext> is h5 in a build with HDF5 when config.h5 exists, else gfr (the raw
// container of gfb_files.h, same dataset and attribute names).
//
// Differences from the reference, all deliberate:
//  * --resume reads the restart file before the restart writer truncates it
//    (the reference creates the writer first, solver.cpp:349-357 before
//    365-384, so its resume always starts from step 0);
//  * output directories are created as needed (the reference's restart
//    writer needs wavefields/ to exist, restart.cpp:91-95);
//  * GFB_PRECISION=fp32 in the environment selects the FP32 element path
//    (FP64 otherwise, the reference's arithmetic).
#include <sys/stat.h>
#include <sys/types.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gfb.h"
#include "gfb_files.h"
#include "gfb_internal.h"

namespace {

using gfb::files::Reader;
using gfb::files::Type;
using gfb::files::Writer;

bool file_exists(const std::string& p) {
    struct stat st;
    return ::stat(p.c_str(), &st) == 0;
}

void make_dirs(const std::string& path) {
    std::string cur;
    std::stringstream ss(path);
    std::string part;
    while (std::getline(ss, part, '/')) {
        if (part.empty()) continue;
        cur += (cur.empty() ? "" : "/") + part;
        ::mkdir(cur.c_str(), 0755);
    }
}

// Timestamped log file log/forward_{dir}_{rank}.log, truncated at start;
// info lines echoed to stdout, errors to stderr (logger.hpp:23-135).
class Logger {
public:
    Logger(const std::string& direction, int rank) {
        ::mkdir("log", 0755);
        const std::string name = "log/forward_" + direction + "_" + std::to_string(rank) + ".log";
        file_.open(name, std::ios::out | std::ios::trunc);
        if (!file_.is_open()) std::cerr << "[Rank 0] WARNING: Cannot open log file: " << name << std::endl;
    }
    void info(const std::string& m) {
        write("INFO", m);
        std::cout << "gf_solver: " << m << std::endl;
    }
    void debug(const std::string& m) { write("DEBUG", m); }
    void error(const std::string& m) {
        write("ERROR", m);
        std::cerr << "[Rank 0] " << m << std::endl;
    }
    void progress(const std::string& m) {
        if (file_.is_open()) file_ << stamp() << " [PROG] " << m << std::endl;
        if (FILE* tty = std::fopen("/dev/tty", "w")) {
            std::fputs("\r\x1b[K", tty);
            std::fputs(m.c_str(), tty);
            std::fclose(tty);
        }
    }
    void progress_done() {
        if (FILE* tty = std::fopen("/dev/tty", "w")) {
            std::fputc('\n', tty);
            std::fclose(tty);
        }
    }

private:
    std::ofstream file_;
    static std::string stamp() {
        const auto now = std::chrono::system_clock::now();
        const std::time_t t = std::chrono::system_clock::to_time_t(now);
        const long ms = (long)(std::chrono::duration_cast<std::chrono::milliseconds>(now.time_since_epoch()).count() %
                               1000);
        char buf[32];
        std::tm tmv;
        localtime_r(&t, &tmv);
        std::strftime(buf, sizeof(buf), "%Y-%m-%d %H:%M:%S", &tmv);
        char out[48];
        std::snprintf(out, sizeof(out), "%s.%03ld", buf, ms);
        return out;
    }
    void write(const char* level, const std::string& m) {
        if (!file_.is_open()) return;
        file_ << stamp() << " [" << std::setw(5) << std::setfill(' ') << level << "] " << m << std::endl;
    }
};

// ConfigData of types.hpp:104-140, read as read_config does (io.cpp:577-709).
struct Config {
    std::string title = "untitled";
    int polynomial_order = 3;
    double solver_dt = 0.0, output_dt_s = 0.0;
    int snapshot_stride = 1, nsteps = 0;
    double cfl_safety = 1.0;
    std::string snapshot_precision = "float64";
    double record_depth_max_m = 0.0, record_depth_actual_m = 0.0;
    int log_stride = 1;
    double restart_dt_s = 0.0;
    int restart_stride = 0;
    std::vector<double> stf_t, stf_values;
    std::vector<int64_t> src_cell_ids;
    std::vector<double> src_weights;
};

bool read_config(const Reader& r, Config& c, std::string& err) {
    if (r.has_group("/simulation")) {
        const std::string g = "/simulation";
        r.attr_str(g, "title", c.title);
        int po = 0;
        c.polynomial_order = (r.attr_i32(g, "polynomial_order", po) && po > 0) ? po : 3;
        if (!r.attr_f64(g, "solver_dt", c.solver_dt)) {
            err = "Missing required /simulation attribute: solver_dt";
            return false;
        }
        if (!r.attr_f64(g, "output_dt_s", c.output_dt_s)) c.output_dt_s = c.solver_dt;
        if (!r.attr_i32(g, "snapshot_stride", c.snapshot_stride)) c.snapshot_stride = 1;
        if (!r.attr_i32(g, "nsteps", c.nsteps)) {
            err = "Missing required /simulation attribute: nsteps";
            return false;
        }
        r.attr_f64(g, "cfl_safety", c.cfl_safety);
        r.attr_str(g, "snapshot_precision", c.snapshot_precision);
        r.attr_f64(g, "record_depth_max_m", c.record_depth_max_m);
        r.attr_f64(g, "record_depth_actual_m", c.record_depth_actual_m);
        r.attr_f64(g, "restart_dt_s", c.restart_dt_s);
        r.attr_i32(g, "restart_stride", c.restart_stride);
        r.attr_i32(g, "log_stride", c.log_stride);
    } else {
        // legacy flat datasets (io.cpp:628-648)
        std::vector<double> v;
        c.polynomial_order = r.read_f64("polynomial_order", v) && !v.empty() ? (int)v[0] : 3;
        c.solver_dt = r.read_f64("dt", v) && !v.empty() ? v[0] : 0.005;
        c.output_dt_s = c.solver_dt;
        c.nsteps = r.read_f64("nsteps", v) && !v.empty() ? (int)v[0] : 1000;
        c.cfl_safety = r.read_f64("cfl_safety", v) && !v.empty() ? v[0] : 1.0;
        c.snapshot_stride = 1;
        std::vector<int64_t> f32;
        c.snapshot_precision = (r.read_i64("use_float32", f32) && !f32.empty() && f32[0] == 1) ? "float32" : "float64";
    }
    if (r.has_group("/source")) {
        r.read_f64("/source/stf_t", c.stf_t);
        r.read_f64("/source/stf_values", c.stf_values);
    } else {
        r.read_f64("stf_t", c.stf_t);
        r.read_f64("stf_values", c.stf_values);
    }
    r.read_i64("/source/cells/cell_ids", c.src_cell_ids);
    r.read_f64("/source/cells/weights", c.src_weights);
    if (c.log_stride < 1) c.log_stride = 1;
    return true;
}

// RankData of types.hpp:27-100, the fields the time loop reads.
struct Partition {
    int n_cell = 0, ngll = 0, n_rank_node = 0;
    std::vector<int64_t> local_cell_ids;
    std::vector<double> jacobian, dxi_dx, mass, density, lambda_, mu, damping;
    std::vector<int32_t> pml_region;
    std::vector<double> pml_coef_alpha, pml_coef_abar;
    std::vector<int32_t> ibool;  // merged: local_cell2global_node of every partition
    bool has_recording = false;
    std::vector<int64_t> gll_node_ids, rec_cell_global;
    std::vector<double> gll_node_coords;
    std::vector<int32_t> rec_cell_local, cell_gll_node_index;
};

// read_partition (io.cpp:182-317), the datasets the merged time loop uses.
bool read_partition(const Reader& r, const std::string& path, Partition& p, std::string& err) {
    if (!r.read_i64("/partition/local_cell_ids", p.local_cell_ids)) {
        err = path + ": missing /partition/local_cell_ids";
        return false;
    }
    p.n_cell = (int)p.local_cell_ids.size();
    const auto cd = r.dims("/field/cell/coords");
    p.ngll = cd.size() >= 4 ? (int)cd[1] : 5;
    r.read_f64("/field/cell/jacobian", p.jacobian);
    r.read_f64("/field/cell/dxi_dx", p.dxi_dx);
    r.read_f64("/field/cell/mass", p.mass);
    r.read_f64("/field/cell/density", p.density);
    r.read_f64("/field/cell/lambda", p.lambda_);
    r.read_f64("/field/cell/mu", p.mu);
    r.read_f64("/field/cell/damping", p.damping);
    r.read_i32("/field/cell/pml_region", p.pml_region);
    r.read_f64("/field/cell/pml_coef_alpha", p.pml_coef_alpha);
    r.read_f64("/field/cell/pml_coef_abar", p.pml_coef_abar);
    r.read_i32("/field/cell/local_cell2global_node", p.ibool);
    r.attr_i32("/field/cell", "n_rank_node", p.n_rank_node);
    if (r.has_group("/recording")) {
        p.has_recording = true;
        if (!r.read_i64("/recording/gll_node_ids", p.gll_node_ids) ||
            !r.read_f64("/recording/gll_node_coords", p.gll_node_coords) ||
            !r.read_i32("/recording/rec_cell_local", p.rec_cell_local) ||
            !r.read_i32("/recording/cell_gll_node_index", p.cell_gll_node_index) ||
            !r.read_i64("/recording/rec_cell_global_ids", p.rec_cell_global)) {
            err = path + ": incomplete /recording group";
            return false;
        }
    }
    return true;
}

template <typename T>
void append(std::vector<T>& a, const std::vector<T>& b) {
    a.insert(a.end(), b.begin(), b.end());
}

// read_partition_all (io.cpp:319-450): partitions 0..R-1 concatenated in
// order; the merged node numbering is the concatenated
// local_cell2global_node (global ids agree across partitions); recording
// nodes deduplicated by global id in first-seen order, rec_cell_local
// offset by the cells of the earlier partitions, cell_gll_node_index
// remapped to the merged node list; n_rank_node = max id + 1.
bool read_partition_all(const std::string& dir, const std::string& ext, Partition& m, int& n_partitions,
                        std::string& err) {
    n_partitions = 0;
    while (file_exists(dir + "/partition_" + std::to_string(n_partitions) + "." + ext)) ++n_partitions;
    if (n_partitions == 0) {
        err = "read_partition_all: no partition files found in " + dir;
        return false;
    }
    std::unordered_map<int64_t, int32_t> node_index;
    int cumulative = 0;
    for (int r = 0; r < n_partitions; ++r) {
        const std::string path = dir + "/partition_" + std::to_string(r) + "." + ext;
        auto rd = gfb::files::open_reader(path, err);
        if (!rd) return false;
        Partition p;
        if (!read_partition(*rd, path, p, err)) return false;
        if (r > 0 && p.ngll != m.ngll) {
            err = "read_partition_all: partition " + std::to_string(r) + " has NGLL=" + std::to_string(p.ngll) +
                  " but expected " + std::to_string(m.ngll);
            return false;
        }
        if (r == 0) {
            m = std::move(p);
            cumulative = m.n_cell;
            for (size_t i = 0; i < m.gll_node_ids.size(); ++i) node_index[m.gll_node_ids[i]] = (int32_t)i;
            continue;
        }
        append(m.local_cell_ids, p.local_cell_ids);
        append(m.jacobian, p.jacobian);
        append(m.dxi_dx, p.dxi_dx);
        append(m.mass, p.mass);
        append(m.density, p.density);
        append(m.lambda_, p.lambda_);
        append(m.mu, p.mu);
        append(m.damping, p.damping);
        append(m.pml_region, p.pml_region);
        append(m.pml_coef_alpha, p.pml_coef_alpha);
        append(m.pml_coef_abar, p.pml_coef_abar);
        append(m.ibool, p.ibool);
        if (p.has_recording) {
            m.has_recording = true;
            std::vector<int32_t> to_merged(p.gll_node_ids.size());
            for (size_t i = 0; i < p.gll_node_ids.size(); ++i) {
                auto it = node_index.find(p.gll_node_ids[i]);
                if (it == node_index.end()) {
                    const int32_t k = (int32_t)m.gll_node_ids.size();
                    node_index[p.gll_node_ids[i]] = k;
                    m.gll_node_ids.push_back(p.gll_node_ids[i]);
                    for (int d = 0; d < 3; ++d) m.gll_node_coords.push_back(p.gll_node_coords[i * 3 + d]);
                    to_merged[i] = k;
                } else {
                    to_merged[i] = it->second;
                }
            }
            append(m.rec_cell_global, p.rec_cell_global);
            for (int32_t c : p.rec_cell_local) m.rec_cell_local.push_back(c + cumulative);
            for (int32_t q : p.cell_gll_node_index) {
                if (q < 0 || (size_t)q >= to_merged.size()) {
                    err = path + ": cell_gll_node_index entry out of range";
                    return false;
                }
                m.cell_gll_node_index.push_back(to_merged[q]);
            }
        }
        cumulative += p.n_cell;
    }
    m.n_cell = cumulative;
    if (m.ibool.empty()) {
        err = "read_partition_all: the partitions carry no /field/cell/local_cell2global_node";
        return false;
    }
    m.n_rank_node = *std::max_element(m.ibool.begin(), m.ibool.end()) + 1;
    return true;
}

// Restart file wavefields/{dir}/restart_0.<ext>: created (truncated) with
// its attributes at start; each write replaces step, time_s and the state
// (restart.cpp:87-139, global-DOF layout).
class RestartFile {
public:
    RestartFile(std::string path, std::string dir, int ngll, int n_node)
        : path_(std::move(path)), dir_(std::move(dir)), ngll_(ngll), n_node_(n_node) {}
    bool write(int step, double time_s, const std::vector<double>* u, const std::vector<double>* v,
               const std::vector<double>* a, const std::vector<double>* damping, std::string& err) {
        auto w = gfb::files::create_writer(path_, err);
        if (!w) return false;
        w->attr_str("/", "source_direction", dir_);
        w->attr_i32("/", "rank", 0);
        w->attr_i32("/", "ngll", ngll_);
        w->attr_i32("/", "use_global_dof", 1);
        w->attr_i32("/", "n_rank_node", n_node_);
        if (u) {
            w->attr_i32("/", "step", step);
            w->attr_f64("/", "time_s", time_s);
            const std::vector<uint64_t> ds{(uint64_t)n_node_ * 3}, dd{(uint64_t)n_node_};
            w->dataset("displacement", Type::F64, ds, u->data());
            w->dataset("velocity", Type::F64, ds, v->data());
            w->dataset("acceleration", Type::F64, ds, a->data());
            w->dataset("pml_damping", Type::F64, dd, damping->data());
        }
        return w->close(err);
    }

private:
    std::string path_, dir_;
    int ngll_, n_node_;
};

// Restart state saved by an earlier run (read_restart, restart.cpp:141-200).
bool read_restart(const std::string& path, int n_node, int& step, std::vector<double>& u, std::vector<double>& v,
                  std::vector<double>& a, std::string& err) {
    auto r = gfb::files::open_reader(path, err);
    if (!r) return false;
    if (!r->attr_i32("/", "step", step) || !r->read_f64("displacement", u) || !r->read_f64("velocity", v) ||
        !r->read_f64("acceleration", a)) {
        err = "no saved state in " + path;
        return false;
    }
    const size_t n = (size_t)n_node * 3;
    if (u.size() != n || v.size() != n || a.size() != n) {
        err = path + ": state size does not match the mesh";
        return false;
    }
    return true;
}

// One snapshot file (RecordWriter::write_step, record.cpp:175-257).
struct RecordMeta {
    std::string dir;
    int ngll = 0, n_rec = 0;
    bool f32 = false;
    double depth_max = 0.0, depth_actual = 0.0;
    const Partition* p = nullptr;
};

bool write_record(const std::string& path, const RecordMeta& M, int step, const void* strain, const void* u,
                  const void* v, const void* a, std::string& err) {
    auto w = gfb::files::create_writer(path, err);
    if (!w) return false;
    const Partition& p = *M.p;
    const uint64_t nn = (uint64_t)M.ngll * M.ngll * M.ngll;
    w->attr_str("/", "source_direction", M.dir);
    w->attr_i32("/", "rank", 0);
    w->attr_i32("/", "ngll", M.ngll);
    w->attr_str("/", "basis", "gll");
    w->attr_i32("/", "n_rec_cell", M.n_rec);
    w->attr_i32("/", "n_unique_gll", (int)p.gll_node_ids.size());
    w->attr_bool("/", "excludes_pml", p.has_recording);
    w->attr_f64("/", "record_depth_max_m", M.depth_max);
    w->attr_f64("/", "record_depth_actual_m", M.depth_actual);
    if (!p.gll_node_ids.empty()) {
        w->dataset("gll_node_ids", Type::I64, {p.gll_node_ids.size()}, p.gll_node_ids.data());
        w->dataset("gll_node_coords", Type::F64, {p.gll_node_ids.size(), 3}, p.gll_node_coords.data());
    }
    w->dataset("cell_gll_node_index", Type::I32, {(uint64_t)M.n_rec, nn}, p.cell_gll_node_index.data());
    if (!p.rec_cell_global.empty())
        w->dataset("recording_cell_model_index", Type::I64, {(uint64_t)M.n_rec}, p.rec_cell_global.data());
    const Type t = M.f32 ? Type::F32 : Type::F64;
    w->dataset("strain", t, {1, (uint64_t)M.n_rec, nn, 6}, strain, true);
    w->dataset("displacement", t, {1, (uint64_t)M.n_rec, nn, 3}, u, true);
    w->dataset("velocity", t, {1, (uint64_t)M.n_rec, nn, 3}, v, true);
    w->dataset("acceleration", t, {1, (uint64_t)M.n_rec, nn, 3}, a, true);
    (void)step;
    return w->close(err);
}

std::string fmt_double(double x) {
    return std::to_string(x);
}

int run(const std::string& direction, bool resume) {
    Logger log(direction, 0);
    log.info("single process, direction=" + direction);
    try {
        const bool h5 = gfb::files::have_hdf5() && file_exists("config.h5");
        const std::string ext = h5 ? "h5" : "gfr";
        const std::string config_path = "config." + ext;
        std::string err;
        auto t_io = std::chrono::steady_clock::now();
        auto cr = gfb::files::open_reader(config_path, err);
        if (!cr) throw std::runtime_error(err);
        Config cfg;
        if (!read_config(*cr, cfg, err)) throw std::runtime_error(err);
        cr.reset();
        const int ngll = cfg.polynomial_order + 1;
        auto secs = [](std::chrono::steady_clock::time_point t0) {
            return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        };
        log.debug("  config read: " + fmt_double(secs(t_io)) + "s");
        log.debug("  polynomial_order=" + std::to_string(cfg.polynomial_order) + " ngll=" + std::to_string(ngll));
        log.debug("  solver_dt=" + fmt_double(cfg.solver_dt) + " nsteps=" + std::to_string(cfg.nsteps));
        log.debug("  snapshot_stride=" + std::to_string(cfg.snapshot_stride) +
                  " precision=" + cfg.snapshot_precision);

        t_io = std::chrono::steady_clock::now();
        Partition part;
        int n_parts = 0;
        if (!read_partition_all("partitions", ext, part, n_parts, err)) throw std::runtime_error(err);
        log.debug("  merged " + std::to_string(part.n_cell) + " elements from all partitions");
        log.debug("  partition read: " + fmt_double(secs(t_io)) + "s");
        if (part.ngll != ngll)
            throw std::runtime_error("partition NGLL " + std::to_string(part.ngll) +
                                     " does not match polynomial_order " + std::to_string(cfg.polynomial_order));
        const size_t nn = (size_t)ngll * ngll * ngll;
        log.info("  n_local_cell=" + std::to_string(part.n_cell) + " n_gll_per_elem=" + std::to_string(nn) +
                 " n_rank_node=" + std::to_string(part.n_rank_node));

        gfb_mesh m{};
        m.n_cell = part.n_cell;
        m.ngll = ngll;
        m.n_node = part.n_rank_node;
        m.ibool = part.ibool.data();
        m.cell_ids = part.local_cell_ids.data();
        m.dxi_dx = part.dxi_dx.data();
        m.jacobian = part.jacobian.data();
        m.lambda_ = part.lambda_.data();
        m.mu = part.mu.data();
        m.density = part.density.empty() ? nullptr : part.density.data();
        m.mass = part.mass.data();
        m.damping = part.damping.empty() ? nullptr : part.damping.data();
        const bool cpml = !part.pml_coef_abar.empty();
        m.pml_region = cpml && !part.pml_region.empty() ? part.pml_region.data() : nullptr;
        m.pml_coef_alpha = cpml ? part.pml_coef_alpha.data() : nullptr;
        m.pml_coef_abar = cpml ? part.pml_coef_abar.data() : nullptr;
        const bool recording = part.has_recording && !part.gll_node_ids.empty();
        if (recording && (part.cell_gll_node_index.size() != part.rec_cell_local.size() * nn ||
                          part.gll_node_coords.size() != part.gll_node_ids.size() * 3 ||
                          (!part.rec_cell_global.empty() && part.rec_cell_global.size() != part.rec_cell_local.size())))
            throw std::runtime_error("recording map sizes disagree (cells, cell_gll_node_index, gll_node_coords)");
        m.n_rec_cell = recording ? (int)part.rec_cell_local.size() : 0;
        m.rec_cell_local = recording ? part.rec_cell_local.data() : nullptr;

        gfb_config c{};
        c.dt = cfg.solver_dt;
        c.snapshot_stride = cfg.snapshot_stride;
        const char* prec = std::getenv("GFB_PRECISION");
        c.precision = (prec && std::strcmp(prec, "fp32") == 0) ? GFB_FP32 : GFB_FP64;
        c.n_field = 1;
        c.field_dir[0] = direction == "x" ? 0 : (direction == "y" ? 1 : 2);
        c.device = 0;
        c.record_slots = 8;
        const bool f32 = cfg.snapshot_precision == "float32";
        c.flags = f32 ? GFB_FLAG_RECORD_F32 : 0;

        gfb_source src{};
        src.n_src_cell = (int32_t)cfg.src_cell_ids.size();
        src.cell_ids = cfg.src_cell_ids.data();
        src.weights = cfg.src_weights.data();
        src.n_stf = (int32_t)cfg.stf_values.size();
        src.stf = cfg.stf_values.data();
        if (src.n_src_cell > 0 && cfg.src_weights.size() != (size_t)src.n_src_cell * nn)
            throw std::runtime_error("/source/cells/weights does not hold n_src_cell x ngll^3 values");
        if (src.n_src_cell > 0) log.debug("  source elements: " + std::to_string(src.n_src_cell));

        gfb_solver* s = nullptr;
        if (gfb_create(&m, &c, &src, &s) != GFB_OK) throw std::runtime_error(gfb_last_error());
        std::unique_ptr<gfb_solver, gfb_status (*)(gfb_solver*)> guard(s, gfb_destroy);
        // host copies of the merged inputs are no longer needed
        const std::vector<double> damping_node = [&] {
            std::vector<double> d((size_t)part.n_rank_node, 0.0);
            if (!part.damping.empty())
                for (size_t q = 0; q < part.ibool.size(); ++q) d[(size_t)part.ibool[q]] = part.damping[q];
            return d;
        }();
        for (auto* v : {&part.dxi_dx, &part.jacobian, &part.lambda_, &part.mu, &part.density, &part.mass,
                        &part.damping, &part.pml_coef_alpha, &part.pml_coef_abar})
            std::vector<double>().swap(*v);
        log.debug("  record cells: " + std::to_string(m.n_rec_cell));

        const int n_snap = cfg.snapshot_stride > 0 ? cfg.nsteps / cfg.snapshot_stride : 0;
        log.info("  snapshots: " + std::to_string(n_snap) + " (stride=" + std::to_string(cfg.snapshot_stride) +
                 ")" + "  total sim time: " + fmt_double(cfg.nsteps * cfg.solver_dt) + " s");

        int restart_stride = 0;
        if (cfg.restart_dt_s > 0.0 && cfg.solver_dt > 0.0)
            restart_stride = std::max(1, (int)std::lround(cfg.restart_dt_s / cfg.solver_dt));
        else if (cfg.restart_stride > 0)
            restart_stride = cfg.restart_stride;
        const std::string out_dir = "wavefields/" + direction;
        make_dirs(out_dir);
        const std::string restart_path = out_dir + "/restart_0." + ext;

        int start_step = 0;
        if (resume) {
            int rstep = 0;
            std::vector<double> u, v, a;
            if (read_restart(restart_path, part.n_rank_node, rstep, u, v, a, err)) {
                if (rstep > 0 && rstep < cfg.nsteps) {
                    start_step = rstep + 1;
                    if (gfb_set_state(s, 0, start_step, u.data(), v.data(), a.data()) != GFB_OK)
                        throw std::runtime_error(gfb_last_error());
                    log.info("  resumed at step " + std::to_string(start_step) +
                             " (time_s=" + fmt_double(rstep * cfg.solver_dt) + ")");
                }
            } else {
                log.error("  resume failed: " + err + " — starting from scratch");
            }
        }
        RestartFile restart(restart_path, direction, ngll, part.n_rank_node);
        if (!restart.write(0, 0.0, nullptr, nullptr, nullptr, nullptr, err)) throw std::runtime_error(err);
        if (restart_stride > 0) log.info("  restart stride: " + std::to_string(restart_stride));
        else log.debug("  restart: disabled");

        // snapshot files written by a second thread while the steps run
        RecordMeta M;
        M.dir = direction;
        M.ngll = ngll;
        M.n_rec = m.n_rec_cell;
        M.f32 = f32;
        M.depth_max = cfg.record_depth_max_m;
        M.depth_actual = cfg.record_depth_actual_m;
        M.p = &part;
        std::atomic<bool> stepping{true};
        std::string writer_err;
        std::thread writer([&] {
            const size_t nrec = (size_t)M.n_rec * nn, es = f32 ? 4 : 8;
            std::vector<char> st(nrec * 6 * es), u(nrec * 3 * es), v(nrec * 3 * es), a(nrec * 3 * es);
            for (;;) {
                int32_t pending = 0;
                if (gfb_records_pending(s, &pending) != GFB_OK) {
                    writer_err = gfb_last_error();
                    return;
                }
                if (pending == 0) {
                    if (!stepping.load()) return;
                    std::this_thread::sleep_for(std::chrono::microseconds(200));
                    continue;
                }
                int32_t step = 0;
                const gfb_status rs =
                    f32 ? gfb_read_record_f32(s, 0, &step, (float*)st.data(), (float*)u.data(), (float*)v.data(),
                                              (float*)a.data(), 1)
                        : gfb_read_record(s, 0, &step, (double*)st.data(), (double*)u.data(), (double*)v.data(),
                                          (double*)a.data(), 1);
                if (rs != GFB_OK) {
                    writer_err = gfb_last_error();
                    return;
                }
                std::string e;
                const std::string path = out_dir + "/record_0_" + std::to_string(step) + "." + ext;
                if (!write_record(path, M, step, st.data(), u.data(), v.data(), a.data(), e)) {
                    writer_err = e;
                    return;
                }
            }
        });
        auto stop_writer = [&] {
            stepping = false;
            writer.join();
        };

        const auto t_start = std::chrono::steady_clock::now();
        int step = start_step;
        try {
            while (step < cfg.nsteps) {
                // advance to the next step that needs the host: a restart
                // write, a progress line or the end
                int next = cfg.nsteps;
                if (restart_stride > 0) {
                    int r = (step / restart_stride) * restart_stride;
                    if (r < step || r == 0) r += restart_stride;
                    next = std::min(next, r + 1);
                }
                const int ls = cfg.log_stride;
                next = std::min(next, ((step / ls) + 1) * ls);
                next = std::min(next, step + 1000);
                if (gfb_advance(s, next - step) != GFB_OK) throw std::runtime_error(gfb_last_error());
                if (!writer_err.empty()) throw std::runtime_error(writer_err);
                const int last = next - 1;  // the last step done
                if (restart_stride > 0 && last > 0 && last % restart_stride == 0) {
                    std::vector<double> u((size_t)part.n_rank_node * 3), v(u.size()), a(u.size());
                    if (gfb_get_state(s, 0, u.data(), v.data(), a.data()) != GFB_OK)
                        throw std::runtime_error(gfb_last_error());
                    if (!restart.write(last, last * cfg.solver_dt, &u, &v, &a, &damping_node, err))
                        throw std::runtime_error(err);
                }
                for (int k = step; k <= last; ++k) {
                    if ((k + 1) % ls != 0 && k != cfg.nsteps - 1) continue;
                    if (gfb_synchronize(s) != GFB_OK) throw std::runtime_error(gfb_last_error());
                    const double el = secs(t_start);
                    const int pct = (int)((long long)(k + 1) * 100 / cfg.nsteps);
                    const double eta = (k + 1 < cfg.nsteps) ? el * (cfg.nsteps - k - 1) / (k + 1) : 0.0;
                    const std::time_t ft =
                        std::chrono::system_clock::to_time_t(std::chrono::system_clock::now() +
                                                             std::chrono::duration_cast<std::chrono::system_clock::duration>(
                                                                 std::chrono::duration<double>(eta)));
                    char fb[20];
                    std::tm tmv;
                    localtime_r(&ft, &tmv);
                    std::strftime(fb, sizeof(fb), "%Y-%m-%d %H:%M:%S", &tmv);
                    std::ostringstream pr;
                    pr << std::setw(7) << std::left << (std::to_string(k + 1) + "/" + std::to_string(cfg.nsteps))
                       << " " << std::setw(4) << pct << "%" << " elapsed=" << std::fixed << std::setprecision(1)
                       << std::setw(6) << el << "s  eta=" << std::setw(6) << eta << "s" << "  finish~" << fb;
                    log.progress(pr.str());
                }
                step = next;
            }
            if (gfb_synchronize(s) != GFB_OK) throw std::runtime_error(gfb_last_error());
        } catch (...) {
            stop_writer();
            throw;
        }
        stop_writer();
        if (!writer_err.empty()) throw std::runtime_error(writer_err);
        log.progress_done();
        log.info("simulation complete, " + std::to_string(cfg.nsteps) + " steps in " + fmt_double(secs(t_start)) +
                 "s");
    } catch (const std::exception& ex) {
        log.error(std::string("Error: ") + ex.what());
        gfb::set_error(GFB_ERR_IO, ex.what());
        return 1;
    }
    return 0;
}

}  // namespace

extern "C" {

gfb_status gfb_merge_partitions(const char* partition_dir, const char* extension, const char* out_path) {
    if (!partition_dir || !extension || !out_path) return gfb::set_error(GFB_ERR_INVALID, "NULL argument");
    Partition m;
    int n = 0;
    std::string err;
    if (!read_partition_all(partition_dir, extension, m, n, err)) return gfb::set_error(GFB_ERR_IO, err.c_str());
    auto w = gfb::files::create_writer(out_path, err);
    if (!w) return gfb::set_error(GFB_ERR_IO, err.c_str());
    const uint64_t nn = (uint64_t)m.ngll * m.ngll * m.ngll, nc = (uint64_t)m.n_cell;
    w->attr_i32("/", "n_partitions", n);
    w->attr_i32("/", "n_cell", m.n_cell);
    w->attr_i32("/", "ngll", m.ngll);
    w->attr_i32("/", "n_rank_node", m.n_rank_node);
    w->dataset("local_cell_ids", Type::I64, {nc}, m.local_cell_ids.data());
    w->dataset("local_cell2rank_node", Type::I32, {nc, nn}, m.ibool.data());
    auto f64 = [&](const char* name, const std::vector<double>& v) {
        if (!v.empty()) w->dataset(name, Type::F64, {v.size()}, v.data());
    };
    f64("jacobian", m.jacobian);
    f64("dxi_dx", m.dxi_dx);
    f64("mass", m.mass);
    f64("density", m.density);
    f64("lambda", m.lambda_);
    f64("mu", m.mu);
    f64("damping", m.damping);
    f64("pml_coef_alpha", m.pml_coef_alpha);
    f64("pml_coef_abar", m.pml_coef_abar);
    if (!m.pml_region.empty()) w->dataset("pml_region", Type::I32, {m.pml_region.size()}, m.pml_region.data());
    if (m.has_recording) {
        w->dataset("recording/gll_node_ids", Type::I64, {m.gll_node_ids.size()}, m.gll_node_ids.data());
        w->dataset("recording/gll_node_coords", Type::F64, {m.gll_node_coords.size()}, m.gll_node_coords.data());
        w->dataset("recording/rec_cell_local", Type::I32, {m.rec_cell_local.size()}, m.rec_cell_local.data());
        w->dataset("recording/rec_cell_global_ids", Type::I64, {m.rec_cell_global.size()}, m.rec_cell_global.data());
        w->dataset("recording/cell_gll_node_index", Type::I32, {m.cell_gll_node_index.size()},
                   m.cell_gll_node_index.data());
    }
    if (!w->close(err)) return gfb::set_error(GFB_ERR_IO, err.c_str());
    return GFB_OK;
}

int32_t gfb_run_forward(const char* direction, int32_t resume, int32_t effective_nprocs) {
    (void)effective_nprocs;  // one process holds every partition
    if (!direction || (std::strcmp(direction, "x") && std::strcmp(direction, "y") && std::strcmp(direction, "z"))) {
        gfb::set_error(GFB_ERR_INVALID, "--direction must be x, y, or z");
        return 1;
    }
    return run(direction, resume != 0);
}

}  // extern "C"
