// CabanaDEM_B200.hpp -- C++ interface with the reference's class names, over the C ABI of
// libb200dem.so (b200dem.h).  A CabanaDEM example ports by swapping the include and the
// Kokkos lambdas for ordinary lambdas:
//
//   reference (CabanaDEM.hpp)                       here
//   CabanaDEM::Inputs (Input.hpp:41-82)             CabanaDEM::Inputs (flat JSON reader)
//   CabanaDEM::Particles<Mem,3,MaxCnts,MaxWalls>    same template; slices are host mirrors
//     (Particles.hpp:22-297)                        committed by updateParticles()/commit()
//   CabanaDEM::Wall<Mem,3> (Wall.hpp:22-153)         same
//   CabanaDEM::Force<Exec>(cor_pp,cor_pw,mu_pp,mu_pw) same (+ optional quirk bits)
//   CabanaDEM::createSolverDEM<Mem>(...)->run()     same: num_steps + 1 steps
//     (Solver.hpp:66-138)
//   CabanaDEM::Integrator<Exec>(dt).stage1/2/3(p)   Integrator<Solver>(solver).stage1/2/3(p)
//     (Integrator.hpp:15-102)
//   computeForceParticleParticleInfiniteWall(        computeForceParticleParticleInfiniteWall(solver)
//     force, p, wall, neigh, tag, dt) (Force.hpp:700-710)   and solver->buildNeighbors()
//   Particles::output -> particles_<k>.h5            particles_<k>.csv, or .xmf + .bin
//                                                    (setOutputFormat("xdmf"))
//   CabanaBondedDEM::ParticlesBondedDEM<Mem,3,MaxBonds> same template: particle and bond slices,
//     (BondedDEM_Particles.hpp:29-293)              setupBonds<Exec>(), update_mesh_limits, output
//   CabanaBondedDEM::resetForcesAndTorques<Exec>(p), same, one device phase each (the reference's
//     computeBondedForce<Exec>(p, dt),               loop, tst_01_BDEM:295-306, ports unchanged);
//     BondedDEMIntegrator<Exec>(dt).stage1/2/3(p)    ParticlesBondedDEM::run_steps fuses the loop
//     (BondedDEM_Force.hpp:16-348, BondedDEM_Integrator.hpp:15-102)
//
// Slices: slicePosition() etc. return a HostSlice, a shared host copy of one field taken at
// the call; writing through it marks the field dirty, and updateParticles(exec, functor)
// (or commit()) uploads every dirty field.  Reading a slice after a run downloads fresh data.
// Errors throw CabanaDEM::Error with the library's message.
#pragma once

#include <array>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "b200dem.h"

namespace CabanaDEM {

struct DeviceSpace {
    using memory_space = DeviceSpace;
    using execution_space = DeviceSpace;
};
using DefaultExecutionSpace = DeviceSpace;

class Error : public std::runtime_error {
  public:
    explicit Error(const std::string &m) : std::runtime_error(m) {}
};

class Context {
  public:
    explicit Context(int device = 0) {
        if (dem_ctx_create(device, &h_)) throw Error("dem_ctx_create: no usable CUDA device");
    }
    ~Context() { dem_ctx_destroy(h_); }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;
    dem_ctx *handle() const { return h_; }
    void check(int st, const char *what, int allow = 0) const {
        if (st & ~allow) throw Error(std::string(what) + ": " + dem_last_error(h_) + " (status " + std::to_string(st) + ")");
    }
    static std::shared_ptr<Context> get_default() {
        static std::shared_ptr<Context> c = std::make_shared<Context>(0);
        return c;
    }

  private:
    dem_ctx *h_ = nullptr;
};

// ---------------------------------------------------------------------------------------
// Flat JSON reader for {"key": {"value": v, "unit"/"units": u}} (Input.hpp:41-82).
// ---------------------------------------------------------------------------------------
class JsonValue {
  public:
    enum Kind { Null, Number, String, Bool, Array, Object };
    Kind kind = Null;
    double num = 0.0;
    std::string str;
    std::vector<JsonValue> arr;
    std::map<std::string, JsonValue> obj;
    operator double() const { return num; }
    operator int() const { return static_cast<int>(num); }
    const JsonValue &operator[](const std::string &k) const {
        auto it = obj.find(k);
        if (it == obj.end()) throw Error("missing key " + k);
        return it->second;
    }
    const JsonValue &operator[](const char *k) const { return (*this)[std::string(k)]; }
    bool contains(const std::string &k) const { return obj.count(k) != 0; }

    static JsonValue parse(const std::string &text) {
        size_t i = 0;
        JsonValue v = value(text, i);
        return v;
    }

  private:
    static void ws(const std::string &s, size_t &i) {
        while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
    }
    static JsonValue value(const std::string &s, size_t &i) {
        ws(s, i);
        if (i >= s.size()) throw Error("json: unexpected end");
        JsonValue v;
        const char c = s[i];
        if (c == '{') {
            v.kind = Object;
            ++i;
            ws(s, i);
            if (s[i] == '}') { ++i; return v; }
            for (;;) {
                ws(s, i);
                const std::string key = string(s, i);
                ws(s, i);
                if (s[i++] != ':') throw Error("json: expected ':'");
                v.obj[key] = value(s, i);
                ws(s, i);
                if (s[i] == ',') { ++i; continue; }
                if (s[i] == '}') { ++i; break; }
                throw Error("json: expected ',' or '}'");
            }
        } else if (c == '[') {
            v.kind = Array;
            ++i;
            ws(s, i);
            if (s[i] == ']') { ++i; return v; }
            for (;;) {
                v.arr.push_back(value(s, i));
                ws(s, i);
                if (s[i] == ',') { ++i; continue; }
                if (s[i] == ']') { ++i; break; }
                throw Error("json: expected ',' or ']'");
            }
        } else if (c == '"') {
            v.kind = String;
            v.str = string(s, i);
        } else if (s.compare(i, 4, "true") == 0) {
            v.kind = Bool; v.num = 1; i += 4;
        } else if (s.compare(i, 5, "false") == 0) {
            v.kind = Bool; v.num = 0; i += 5;
        } else if (s.compare(i, 4, "null") == 0) {
            i += 4;
        } else {
            v.kind = Number;
            size_t used = 0;
            v.num = std::stod(s.substr(i), &used);
            i += used;
        }
        return v;
    }
    // a JSON string at s[i] ('"' ... '"'), escapes decoded (\uXXXX as UTF-8, surrogate pairs
    // joined); i ends past the closing quote
    static std::string string(const std::string &s, size_t &i) {
        if (i >= s.size() || s[i] != '"') throw Error("json: expected string");
        std::string out;
        for (++i;; ++i) {
            if (i >= s.size()) throw Error("json: unterminated string");
            const char c = s[i];
            if (c == '"') break;
            if (c != '\\') {
                out += c;
                continue;
            }
            if (++i >= s.size()) throw Error("json: unterminated string");
            switch (s[i]) {
                case '"': out += '"'; break;
                case '\\': out += '\\'; break;
                case '/': out += '/'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'n': out += '\n'; break;
                case 'r': out += '\r'; break;
                case 't': out += '\t'; break;
                case 'u': {
                    unsigned cp = hex4(s, i + 1);
                    i += 4;
                    if (cp >= 0xD800 && cp < 0xDC00 && i + 6 < s.size() && s[i + 1] == '\\' && s[i + 2] == 'u') {
                        const unsigned lo = hex4(s, i + 3);
                        if (lo >= 0xDC00 && lo < 0xE000) {
                            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                            i += 6;
                        }
                    }
                    utf8(out, cp);
                    break;
                }
                default: throw Error("json: bad escape");
            }
        }
        ++i;
        return out;
    }
    static unsigned hex4(const std::string &s, size_t at) {
        if (at + 4 > s.size()) throw Error("json: short \\u escape");
        unsigned v = 0;
        for (size_t k = at; k < at + 4; ++k) {
            const char c = s[k];
            v <<= 4;
            if (c >= '0' && c <= '9') v |= unsigned(c - '0');
            else if (c >= 'a' && c <= 'f') v |= unsigned(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= unsigned(c - 'A' + 10);
            else throw Error("json: bad \\u escape");
        }
        return v;
    }
    static void utf8(std::string &out, unsigned cp) {
        if (cp < 0x80) {
            out += char(cp);
        } else if (cp < 0x800) {
            out += char(0xC0 | (cp >> 6));
            out += char(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += char(0xE0 | (cp >> 12));
            out += char(0x80 | ((cp >> 6) & 0x3F));
            out += char(0x80 | (cp & 0x3F));
        } else {
            out += char(0xF0 | (cp >> 18));
            out += char(0x80 | ((cp >> 12) & 0x3F));
            out += char(0x80 | ((cp >> 6) & 0x3F));
            out += char(0x80 | (cp & 0x3F));
        }
    }
};

inline std::vector<std::string> splitString(const std::string &str, char delimiter) {   // Input.hpp:24-38
    std::vector<std::string> result;
    size_t start = 0, end = str.find(delimiter);
    while (end != std::string::npos) {
        result.push_back(str.substr(start, end - start));
        start = end + 1;
        end = str.find(delimiter, start);
    }
    result.push_back(str.substr(start));
    return result;
}

class Inputs {
  public:
    explicit Inputs(const std::string &filename) {
        std::ifstream f(filename);
        if (!f) throw Error("cannot open " + filename);
        std::stringstream ss;
        ss << f.rdbuf();
        inputs_ = JsonValue::parse(ss.str());
        const double tf = inputs_["final_time"]["value"];
        const double dt = inputs_["timestep"]["value"];
        const int num_steps = tf / dt;   // Input.hpp:53, truncation as the reference
        JsonValue ns;
        ns.kind = JsonValue::Object;
        JsonValue v;
        v.kind = JsonValue::Number;
        v.num = num_steps;
        ns.obj["value"] = v;
        inputs_.obj["num_steps"] = ns;
    }
    const JsonValue &operator[](const std::string &label) const { return inputs_[label]["value"]; }
    const JsonValue &operator[](const char *label) const { return (*this)[std::string(label)]; }
    std::string units(const std::string &label) const {
        return inputs_[label].contains("units") ? inputs_[label]["units"].str : std::string();
    }
    bool contains(const std::string &label) const { return inputs_.contains(label); }

  private:
    JsonValue inputs_;
};

// ---------------------------------------------------------------------------------------
// Host mirror of one field.
// ---------------------------------------------------------------------------------------
template <class T>
struct Mirror {
    std::vector<T> data;
    int ncomp = 1;
    bool dirty = false;
    bool fresh = false;
};

template <class T>
class HostSlice {
  public:
    HostSlice() = default;
    explicit HostSlice(std::shared_ptr<Mirror<T>> m) : m_(std::move(m)) {}
    T &operator()(int i, int d = 0) const {
        m_->dirty = true;
        return m_->data[static_cast<size_t>(i) * m_->ncomp + d];
    }
    // read without marking the field for upload
    T get(int i, int d = 0) const { return m_->data[static_cast<size_t>(i) * m_->ncomp + d]; }
    std::size_t size() const { return m_->data.size() / m_->ncomp; }
    const T *data() const { return m_->data.data(); }

  private:
    std::shared_ptr<Mirror<T>> m_;
};

// ---------------------------------------------------------------------------------------
// CSV snapshot: <folder>/particles_<step>.csv, a "# time <t>" line, a header of the reference's
// slice labels with a component suffix and one row per particle, every double with 17
// significant digits (so it reads back bit for bit).  Vectors are [n][3] row-major.
// ---------------------------------------------------------------------------------------
inline void writeCsvSnapshot(const std::string &folder, int step, double time, int n, const double *x,
                             const double *u, const double *w, const double *f, const double *m,
                             const double *rho, const double *r, const int *tc) {
    const std::string path = folder + "/particles_" + std::to_string(step) + ".csv";
    std::FILE *fo = std::fopen(path.c_str(), "w");
    if (!fo) throw Error("cannot write " + path);
    std::fprintf(fo, "# time %.17g\n", time);
    std::fprintf(fo, "id,positions_0,positions_1,positions_2,velocities_0,velocities_1,velocities_2,"
                     "omega_0,omega_1,omega_2,forces_0,forces_1,forces_2,mass,density,radius,"
                     "total_no_tangential_contacts\n");
    for (int i = 0; i < n; ++i)
        std::fprintf(fo, "%d,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,"
                         "%.17g,%.17g,%.17g,%d\n",
                     i, x[3 * i], x[3 * i + 1], x[3 * i + 2], u[3 * i], u[3 * i + 1], u[3 * i + 2], w[3 * i],
                     w[3 * i + 1], w[3 * i + 2], f[3 * i], f[3 * i + 1], f[3 * i + 2], m[i], rho[i], r[i], tc[i]);
    std::fclose(fo);
}

// ---------------------------------------------------------------------------------------
// XDMF snapshot.  The reference's writer (Cabana's HDF5 particle output, called at
// Particles.hpp:306-326) stores one dataset per slice label in particles_<k>.h5 with the
// step's time; viewers open it through an XDMF index.  No HDF5 library is in this image, so
// here the heavy data is one raw little-endian file, particles_<k>.bin (the datasets one after
// another), and particles_<k>.xmf indexes it (XDMF 2: a Polyvertex grid with its Time, the
// positions as XYZ geometry, one node attribute per other dataset, Format="Binary" data items
// with byte offsets), which XDMF readers such as ParaView and VisIt open.
// ---------------------------------------------------------------------------------------
struct XdmfField {
    std::string name;   // dataset name (the reference's slice label)
    const void *data;   // [n][ncomp] row-major
    int ncomp;          // 1 (Scalar attribute) or 3 (Vector; the positions are the Geometry)
    bool is_int;        // int32 instead of float64
};

// <folder>/particles_<step>.xmf and .bin; fields[0] holds the positions.
inline void writeXdmfSnapshot(const std::string &folder, int step, double time, int n,
                              const std::vector<XdmfField> &fields) {
    const unsigned short probe = 1;
    if (*reinterpret_cast<const unsigned char *>(&probe) != 1) throw Error("writeXdmfSnapshot: big-endian host");
    if (fields.empty() || fields[0].ncomp != 3 || fields[0].is_int)
        throw Error("writeXdmfSnapshot: fields[0] must be the positions, [n][3] float64");
    for (const auto &f : fields)
        if (f.ncomp != 1 && f.ncomp != 3) throw Error("writeXdmfSnapshot: " + f.name + ": 1 or 3 components");
    const std::string stem = "particles_" + std::to_string(step);
    const std::string bin = folder + "/" + stem + ".bin", xmf = folder + "/" + stem + ".xmf";
    std::vector<long> seek;
    {
        std::FILE *fb = std::fopen(bin.c_str(), "wb");
        if (!fb) throw Error("cannot write " + bin);
        long at = 0;
        for (const auto &f : fields) {
            const size_t bytes = static_cast<size_t>(n) * f.ncomp * (f.is_int ? 4 : 8);
            seek.push_back(at);
            if (bytes && std::fwrite(f.data, 1, bytes, fb) != bytes) {
                std::fclose(fb);
                throw Error("short write to " + bin);
            }
            at += static_cast<long>(bytes);
        }
        if (std::fclose(fb) != 0) throw Error("cannot close " + bin);
    }
    std::FILE *fx = std::fopen(xmf.c_str(), "w");
    if (!fx) throw Error("cannot write " + xmf);
    auto item = [&](size_t k) {
        const XdmfField &f = fields[k];
        std::fprintf(fx,
                     "        <DataItem Dimensions=\"%d%s\" NumberType=\"%s\" Precision=\"%d\" Format=\"Binary\" "
                     "Endian=\"Little\" Seek=\"%ld\">%s.bin</DataItem>\n",
                     n, f.ncomp == 3 ? " 3" : "", f.is_int ? "Int" : "Float", f.is_int ? 4 : 8, seek[k], stem.c_str());
    };
    std::fprintf(fx, "<?xml version=\"1.0\" ?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n<Xdmf Version=\"2.0\">\n");
    std::fprintf(fx, "  <Domain>\n    <Grid Name=\"particles\" GridType=\"Uniform\">\n");
    std::fprintf(fx, "      <Time Value=\"%.17g\"/>\n", time);
    std::fprintf(fx, "      <Topology TopologyType=\"Polyvertex\" NumberOfElements=\"%d\" NodesPerElement=\"1\"/>\n", n);
    std::fprintf(fx, "      <Geometry GeometryType=\"XYZ\">\n");
    item(0);
    std::fprintf(fx, "      </Geometry>\n");
    for (size_t k = 1; k < fields.size(); ++k) {
        std::fprintf(fx, "      <Attribute Name=\"%s\" AttributeType=\"%s\" Center=\"Node\">\n", fields[k].name.c_str(),
                     fields[k].ncomp == 3 ? "Vector" : "Scalar");
        item(k);
        std::fprintf(fx, "      </Attribute>\n");
    }
    std::fprintf(fx, "    </Grid>\n  </Domain>\n</Xdmf>\n");
    if (std::fclose(fx) != 0) throw Error("cannot close " + xmf);
}

// ---------------------------------------------------------------------------------------
// Particles<MemorySpace, Dim, MaxCnts, MaxNoWalls> (Particles.hpp:22-71)
// ---------------------------------------------------------------------------------------
template <class MemorySpace, int Dimension, int MaxCnts, int MaxNoWalls>
class Particles {
  public:
    static constexpr int dim = Dimension;
    std::array<double, 3> mesh_lo{}, mesh_hi{};   // kept for source compatibility: the device grid
                                                  // follows the particles' bounding box

    template <class ExecSpace>
    Particles(const ExecSpace &, std::size_t n, const std::string &output_folder = "",
              std::shared_ptr<Context> ctx = nullptr)
        : n_(static_cast<int>(n)), out_(output_folder), ctx_(ctx ? ctx : Context::get_default()) {
        ctx_->check(dem_particles_create(ctx_->handle(), n_, MaxCnts, MaxNoWalls, &h_), "dem_particles_create");
        // Particles.hpp:53-61: the output folder is created if it does not exist
        if (!out_.empty()) std::filesystem::create_directories(out_);
        // snapshot format for programs that do not call setOutputFormat (the example drivers)
        if (const char *fmt = std::getenv("CABANADEM_OUTPUT_FORMAT")) setOutputFormat(fmt);
    }
    ~Particles() { dem_particles_destroy(h_); }
    Particles(const Particles &) = delete;
    Particles &operator=(const Particles &) = delete;

    HostSlice<double> slicePosition() { return slice_d(DEM_F_X, 3); }
    HostSlice<double> sliceVelocity() { return slice_d(DEM_F_U, 3); }
    HostSlice<double> sliceOmega() { return slice_d(DEM_F_OMEGA, 3); }
    HostSlice<double> sliceForce() { return slice_d(DEM_F_FORCE, 3); }
    HostSlice<double> sliceTorque() { return slice_d(DEM_F_TORQUE, 3); }
    HostSlice<double> sliceMass() { return slice_d(DEM_F_M, 1); }
    HostSlice<double> sliceDensity() { return slice_d(DEM_F_RHO, 1); }
    HostSlice<double> sliceRadius() { return slice_d(DEM_F_RAD, 1); }
    HostSlice<double> sliceMomentOfInertia() { return slice_d(DEM_F_I, 1); }
    HostSlice<double> sliceYoungsMod() { return slice_d(DEM_F_E, 1); }
    HostSlice<double> slicePoissonsRatio() { return slice_d(DEM_F_NU, 1); }
    HostSlice<double> sliceShearMod() { return slice_d(DEM_F_G, 1); }
    HostSlice<double> sliceTangentialDispSSx() { return slice_d(DEM_F_TNG_SS_X, MaxCnts); }
    HostSlice<double> sliceTangentialDispSSy() { return slice_d(DEM_F_TNG_SS_Y, MaxCnts); }
    HostSlice<double> sliceTangentialDispSSz() { return slice_d(DEM_F_TNG_SS_Z, MaxCnts); }
    HostSlice<double> sliceTangentialDispSWx() { return slice_d(DEM_F_TNG_SW_X, MaxNoWalls); }
    HostSlice<double> sliceTangentialDispSWy() { return slice_d(DEM_F_TNG_SW_Y, MaxNoWalls); }
    HostSlice<double> sliceTangentialDispSWz() { return slice_d(DEM_F_TNG_SW_Z, MaxNoWalls); }
    HostSlice<int> sliceTangentialDispIdx() { return slice_i(DEM_F_TNG_IDX, MaxCnts); }
    // the reference's accelerations (Particles.hpp:117-124) are written by its examples' set-up
    // functors and read by nothing on the path: a host-only [n][3] array here
    HostSlice<double> sliceAcceleration() {
        if (!au_) {
            au_ = std::make_shared<Mirror<double>>();
            au_->ncomp = 3;
            au_->data.assign(static_cast<size_t>(n_) * 3, 0.0);
            au_->fresh = true;
        }
        return HostSlice<double>(au_);
    }
    HostSlice<int> sliceTotalNoTangentialContacts() { return slice_i(DEM_F_TNG_COUNT, 1); }

    // updateParticles(exec, functor) (Particles.hpp:91-97): functor(pid) on the host for every
    // particle, then every slice written through is uploaded.
    template <class ExecSpace, class Functor>
    void updateParticles(const ExecSpace &, const Functor &f) {
        for (int pid = 0; pid < n_; ++pid) f(pid);
        commit();
    }

    void commit() {
        for (auto &kv : md_)
            if (kv.second->dirty) {
                ctx_->check(dem_particles_set(h_, kv.first, kv.second->data.data(), (long)kv.second->data.size()),
                            "dem_particles_set");
                kv.second->dirty = false;
            }
        for (auto &kv : mi_)
            if (kv.second->dirty) {
                ctx_->check(dem_particles_set(h_, kv.first, kv.second->data.data(), (long)kv.second->data.size()),
                            "dem_particles_set");
                kv.second->dirty = false;
            }
    }
    // device -> mirrors (called by the solver after it advances the state)
    void invalidate() {
        for (auto &kv : md_) kv.second->fresh = false;
        for (auto &kv : mi_) kv.second->fresh = false;
    }

    // Snapshot format of output(): "csv" (the default), "xdmf" or "both".  The environment
    // variable CABANADEM_OUTPUT_FORMAT sets it for every particle set a program creates.
    void setOutputFormat(const std::string &format) {
        if (format != "csv" && format != "xdmf" && format != "both")
            throw Error("setOutputFormat: csv, xdmf or both");
        format_ = format;
    }

    // output(step, time) (Particles.hpp:299-346): one snapshot per call, <folder>/particles_<step>.csv,
    // one row per particle with the fields the reference writes to particles_<step>.h5 (its
    // HDF5 writer; no HDF5 library here) minus the accelerations, which are not stored.
    // Columns are named after the reference's slices with a component suffix.  With the
    // "xdmf" format the same datasets go to particles_<step>.xmf / .bin (writeXdmfSnapshot).
    // No folder, no output.
    void output(int output_step, double output_time) {
        if (out_.empty()) return;
        if (format_ != "csv") {
            auto x = slicePosition();
            auto u = sliceVelocity();
            auto w = sliceOmega();
            auto f = sliceForce();
            auto m = sliceMass();
            auto rho = sliceDensity();
            auto r = sliceRadius();
            auto tc = sliceTotalNoTangentialContacts();
            writeXdmfSnapshot(out_, output_step, output_time, n_,
                              {{"positions", x.data(), 3, false}, {"velocities", u.data(), 3, false},
                               {"omega", w.data(), 3, false}, {"forces", f.data(), 3, false},
                               {"mass", m.data(), 1, false}, {"density", rho.data(), 1, false},
                               {"radius", r.data(), 1, false}, {"total_no_tangential_contacts", tc.data(), 1, true}});
            if (format_ == "xdmf") return;
        }
        auto x = slicePosition();
        auto u = sliceVelocity();
        auto w = sliceOmega();
        auto f = sliceForce();
        auto m = sliceMass();
        auto rho = sliceDensity();
        auto r = sliceRadius();
        auto tc = sliceTotalNoTangentialContacts();
        writeCsvSnapshot(out_, output_step, output_time, n_, x.data(), u.data(), w.data(), f.data(), m.data(),
                         rho.data(), r.data(), tc.data());
    }
    const std::string &output_folder() const { return out_; }

    // resize(n) (Particles.hpp:273-297): the first min(n, size()) particles keep their values;
    // added particles start zeroed with empty contact slots (tangential index -1).  The device
    // set is re-created, so no solver may be attached: create solvers after the last resize.
    // Slices taken before the call see the new size.  External forces and fix flags are reset.
    void resize(std::size_t n) {
        if (attached_ > 0) throw Error("Particles::resize: a solver is attached to this particle set");
        const int nn = static_cast<int>(n);
        const int dfields[][2] = {{DEM_F_X, 3},          {DEM_F_U, 3},          {DEM_F_OMEGA, 3},
                                  {DEM_F_FORCE, 3},      {DEM_F_TORQUE, 3},     {DEM_F_M, 1},
                                  {DEM_F_RHO, 1},        {DEM_F_RAD, 1},        {DEM_F_I, 1},
                                  {DEM_F_E, 1},          {DEM_F_NU, 1},         {DEM_F_G, 1},
                                  {DEM_F_TNG_SS_X, MaxCnts}, {DEM_F_TNG_SS_Y, MaxCnts}, {DEM_F_TNG_SS_Z, MaxCnts},
                                  {DEM_F_TNG_SW_X, MaxNoWalls}, {DEM_F_TNG_SW_Y, MaxNoWalls},
                                  {DEM_F_TNG_SW_Z, MaxNoWalls}};
        for (const auto &f : dfields) slice_d(f[0], f[1]);   // current values (or pending edits)
        slice_i(DEM_F_TNG_IDX, MaxCnts);
        slice_i(DEM_F_TNG_COUNT, 1);
        dem_particles *h = nullptr;
        ctx_->check(dem_particles_create(ctx_->handle(), nn, MaxCnts, MaxNoWalls, &h), "dem_particles_create");
        dem_particles_destroy(h_);
        h_ = h;
        n_ = nn;
        for (auto &kv : md_) {
            kv.second->data.resize(static_cast<size_t>(nn) * kv.second->ncomp, 0.0);
            kv.second->dirty = kv.second->ncomp > 0;
            kv.second->fresh = true;
        }
        for (auto &kv : mi_) {
            kv.second->data.resize(static_cast<size_t>(nn) * kv.second->ncomp, kv.first == DEM_F_TNG_IDX ? -1 : 0);
            kv.second->dirty = kv.second->ncomp > 0;
            kv.second->fresh = true;
        }
        if (au_) au_->data.resize(static_cast<size_t>(nn) * 3, 0.0);
        commit();
    }

    // External force added before the pair forces, [n][3], and DEM_FIX_* boundary flags, [n]
    // (the hooks of the reference examples' applyTensileForce / applyBoundaryConditions).
    void setExternalForce(const std::vector<double> &f) {
        ctx_->check(dem_particles_set(h_, DEM_F_EXT_FORCE, f.data(), (long)f.size()), "dem_particles_set");
    }
    void setFixFlags(const std::vector<unsigned char> &flags) {
        ctx_->check(dem_particles_set(h_, DEM_F_FIX, flags.data(), (long)flags.size()), "dem_particles_set");
    }

    // solvers hold the device handle: resize() is refused while one exists
    void attach_solver(int d) { attached_ += d; }

    std::size_t size() const { return static_cast<std::size_t>(n_); }
    dem_particles *handle() { return h_; }
    Context &context() { return *ctx_; }
    std::shared_ptr<Context> context_ptr() { return ctx_; }

  private:
    HostSlice<double> slice_d(int field, int nc) {
        auto &m = md_[field];
        if (!m) {
            m = std::make_shared<Mirror<double>>();
            m->ncomp = nc;
            m->data.assign(static_cast<size_t>(n_) * nc, 0.0);
        }
        if (!m->fresh && !m->dirty && nc > 0) {
            ctx_->check(dem_particles_get(h_, field, m->data.data(), (long)m->data.size()), "dem_particles_get");
            m->fresh = true;
        }
        return HostSlice<double>(m);
    }
    HostSlice<int> slice_i(int field, int nc) {
        auto &m = mi_[field];
        if (!m) {
            m = std::make_shared<Mirror<int>>();
            m->ncomp = nc;
            m->data.assign(static_cast<size_t>(n_) * nc, 0);
        }
        if (!m->fresh && !m->dirty && nc > 0) {
            ctx_->check(dem_particles_get(h_, field, m->data.data(), (long)m->data.size()), "dem_particles_get");
            m->fresh = true;
        }
        return HostSlice<int>(m);
    }

    int n_;
    int attached_ = 0;
    std::string out_;
    std::string format_ = "csv";
    std::shared_ptr<Context> ctx_;
    dem_particles *h_ = nullptr;
    std::map<int, std::shared_ptr<Mirror<double>>> md_;
    std::map<int, std::shared_ptr<Mirror<int>>> mi_;
    std::shared_ptr<Mirror<double>> au_;
};

// ---------------------------------------------------------------------------------------
// Wall<MemorySpace, Dim> (Wall.hpp:22-153)
// ---------------------------------------------------------------------------------------
template <class MemorySpace, int Dimension>
class Wall {
  public:
    template <class ExecSpace>
    Wall(const ExecSpace &, std::size_t n, const std::string & = "", std::shared_ptr<Context> ctx = nullptr)
        : n_(static_cast<int>(n)), ctx_(ctx ? ctx : Context::get_default()) {
        ctx_->check(dem_walls_create(ctx_->handle(), n_, &h_), "dem_walls_create");
        for (int f = DEM_W_X; f <= DEM_W_G; ++f) {
            auto m = std::make_shared<Mirror<double>>();
            m->ncomp = f <= DEM_W_NORMAL ? 3 : 1;
            m->data.assign(static_cast<size_t>(n_) * m->ncomp, 0.0);
            m_[f] = m;
        }
    }
    ~Wall() { dem_walls_destroy(h_); }
    HostSlice<double> slicePosition() { return HostSlice<double>(m_[DEM_W_X]); }
    HostSlice<double> sliceVelocity() { return HostSlice<double>(m_[DEM_W_U]); }
    HostSlice<double> sliceOmega() { return HostSlice<double>(m_[DEM_W_OMEGA]); }
    HostSlice<double> sliceNormal() { return HostSlice<double>(m_[DEM_W_NORMAL]); }
    HostSlice<double> sliceYoungsMod() { return HostSlice<double>(m_[DEM_W_E]); }
    HostSlice<double> slicePoissonsRatio() { return HostSlice<double>(m_[DEM_W_NU]); }
    HostSlice<double> sliceShearMod() { return HostSlice<double>(m_[DEM_W_G]); }
    template <class ExecSpace, class Functor>
    void updateParticles(const ExecSpace &, const Functor &f) {
        for (int pid = 0; pid < n_; ++pid) f(pid);
        commit();
    }
    void commit() {
        for (auto &kv : m_)
            ctx_->check(dem_walls_set(h_, kv.first, kv.second->data.data(), (long)kv.second->data.size()),
                        "dem_walls_set");
    }
    std::size_t size() const { return static_cast<std::size_t>(n_); }
    dem_walls *handle() { return h_; }

  private:
    int n_;
    std::shared_ptr<Context> ctx_;
    dem_walls *h_ = nullptr;
    std::map<int, std::shared_ptr<Mirror<double>>> m_;
};

// Force<ExecutionSpace>(cor_pp, cor_pw, friction_pp, friction_pw) (Force.hpp:16-35)
template <class ExecutionSpace>
class Force {
  public:
    double cor_pp, cor_pw, friction_pp, friction_pw;
    unsigned quirks;
    Force(double cpp, double cpw, double fpp, double fpw, unsigned q = DEM_REF_COMPAT)
        : cor_pp(cpp), cor_pw(cpw), friction_pp(fpp), friction_pw(fpw), quirks(q) {}
    dem_force_params params() const { return dem_force_params{cor_pp, cor_pw, friction_pp, friction_pw, quirks}; }
};

// SolverDEM (Solver.hpp:13-122): the reference rebuilds the neighbour list every step with
// cutoff delta; that is the default here.  set_skin() switches to the Verlet-skin mode.
template <class MemorySpace, class InputType, class ParticleType, class WallType, class ForceModel>
class SolverDEM {
  public:
    SolverDEM(const InputType &inputs, std::shared_ptr<ParticleType> particles, std::shared_ptr<WallType> wall,
              std::shared_ptr<ForceModel> force, double delta, double skin = 0.0, int precision = DEM_FP64,
              std::array<double, 3> gravity = {0.0, 0.0, 0.0})
        : particles_(particles), wall_(wall), force_(force) {
        num_steps = inputs["num_steps"];
        output_frequency = inputs.contains("output_frequency") ? (int)inputs["output_frequency"] : 0;
        dt = inputs["timestep"];
        particles_->commit();
        if (wall_) wall_->commit();
        dem_solver_params sp{};
        sp.dt = dt;
        sp.delta = skin > 0.0 ? 0.0 : delta;
        sp.skin = skin;
        sp.rebuild_every_step = skin > 0.0 ? 0 : 1;
        sp.precision = precision;
        for (int d = 0; d < 3; ++d) sp.gravity[d] = gravity[d];
        const dem_force_params fp = force_->params();
        particles_->context().check(dem_solver_create(particles_->context().handle(), particles_->handle(),
                                                      wall_ ? wall_->handle() : nullptr, &fp, &sp, &h_),
                                    "dem_solver_create");
        particles_->attach_solver(1);
    }
    ~SolverDEM() {
        dem_solver_destroy(h_);
        particles_->attach_solver(-1);
    }

    void set_output(std::function<void(int, double)> f) { out_ = std::move(f); }

    // Solver.hpp:79-97: steps 0..num_steps inclusive, output after every step divisible by
    // output_frequency; the steps between two outputs run as one fused device run
    void run() {
        int step = 0;
        while (step <= num_steps) {
            int stop = num_steps;
            if (output_frequency > 0) {
                const int next_out = (step + output_frequency - 1) / output_frequency * output_frequency;
                if (next_out < stop) stop = next_out;
            }
            run_steps(stop - step + 1);
            output(stop);
            step = stop + 1;
        }
    }
    void run_steps(int n) {
        particles_->commit();
        particles_->context().check(dem_solver_run(h_, n), "dem_solver_run", DEM_ERR_CONTACT_OVERFLOW);
        particles_->invalidate();
    }
    void output(int step) {
        if (output_frequency > 0 && step % output_frequency == 0) {
            std::cout << "We are at " << step << " / " << num_steps << std::endl;
            // Solver.hpp:100-107: particles->output(step / output_frequency, step * dt)
            particles_->output(step / output_frequency, step * dt);
            if (out_) out_(step, step * dt);
        }
    }
    // The reference loop's phases, one launch each, for callers that drive the loop themselves
    // (Solver.hpp:81-94): integrator->stage1 / stage2 (Integrator.hpp:31-74), neighbors->build,
    // computeForceParticleParticleInfiniteWall (Force.hpp:700-710), stage3 (:77-102).  Host
    // edits made through slices are uploaded first; slices read the new state afterwards.
    void stage1() { phase(dem_stage1, "dem_stage1"); }
    void stage2() { phase(dem_stage2, "dem_stage2"); }
    void buildNeighbors() { phase(dem_build_neighbors, "dem_build_neighbors"); }
    void computeForce() { phase(dem_compute_force, "dem_compute_force", DEM_ERR_CONTACT_OVERFLOW); }
    void stage3() { phase(dem_stage3, "dem_stage3"); }

    dem_solver *handle() { return h_; }
    // triangle-mesh wall (dem_solver_set_mesh): tri = nt * 9 vertex coordinates, one material,
    // optional translation velocity (used when the force's DEM_Q6_WALL_STATIC bit is clear)
    void setMesh(const std::vector<double> &tri, double E, double nu, double G,
                 std::array<double, 3> velocity = {0.0, 0.0, 0.0}, int max_contacts = 8) {
        particles_->context().check(dem_solver_set_mesh(h_, tri.empty() ? nullptr : tri.data(), (int)(tri.size() / 9), E,
                                                        nu, G, velocity.data(), max_contacts),
                                    "dem_solver_set_mesh");
    }
    std::array<double, 3> meshTranslation() {
        std::array<double, 3> d{};
        particles_->context().check(dem_solver_mesh_translation(h_, d.data()), "dem_solver_mesh_translation");
        return d;
    }
    // current wall positions [nw][3]: a wall with a velocity moves by dt * u each step when the
    // force's DEM_Q6_WALL_STATIC bit is clear (the reference's walls never move)
    std::vector<double> wallPositions() {
        std::vector<double> x(wall_ ? 3 * wall_->size() : 0);
        particles_->context().check(dem_solver_wall_positions(h_, x.data(), (long)x.size()),
                                    "dem_solver_wall_positions");
        return x;
    }

    int num_steps = 0;
    int output_frequency = 0;
    double dt = 0.0;

  private:
    void phase(int (*f)(dem_solver *), const char *what, int allow = 0) {
        particles_->commit();
        particles_->context().check(f(h_), what, allow);
        particles_->invalidate();
    }

    std::shared_ptr<ParticleType> particles_;
    std::shared_ptr<WallType> wall_;
    std::shared_ptr<ForceModel> force_;
    dem_solver *h_ = nullptr;
    std::function<void(int, double)> out_;
};

// Integrator<ExecutionSpace> (Integrator.hpp:15-102) on a solver's particles: the reference
// constructs it from dt; here the solver holds dt and the device state, so it wraps the solver.
template <class SolverType>
class Integrator {
  public:
    explicit Integrator(std::shared_ptr<SolverType> solver) : s_(std::move(solver)) {}
    template <class ParticleType>
    void stage1(ParticleType &) { s_->stage1(); }
    template <class ParticleType>
    void stage2(ParticleType &) { s_->stage2(); }
    template <class ParticleType>
    void stage3(ParticleType &) { s_->stage3(); }

  private:
    std::shared_ptr<SolverType> s_;
};

// computeForceParticleParticleInfiniteWall (Force.hpp:700-710): zero F and tau, compact the
// tangential contacts, particle-particle force, wall force, on the solver's particles and walls
template <class SolverType>
void computeForceParticleParticleInfiniteWall(SolverType &solver) {
    solver.computeForce();
}

// createSolverDEM<MemorySpace>(inputs, particles, wall, force, delta) (Solver.hpp:127-138)
template <class MemorySpace, class InputsType, class ParticleType, class WallType, class ForceModel>
auto createSolverDEM(const InputsType &inputs, std::shared_ptr<ParticleType> particles,
                     std::shared_ptr<WallType> wall, std::shared_ptr<ForceModel> force, double delta) {
    return std::make_shared<SolverDEM<MemorySpace, InputsType, ParticleType, WallType, ForceModel>>(
        inputs, particles, wall, force, delta);
}

}  // namespace CabanaDEM

namespace CabanaBondedDEM {

using CabanaDEM::Context;
using CabanaDEM::Error;
using CabanaDEM::HostSlice;
using CabanaDEM::Mirror;

// ParticlesBondedDEM<MemorySpace, Dim, MaxBonds> (BondedDEM_Particles.hpp:29-293): the particle
// fields of CabanaDEM::Particles plus the bond slots.  Bond slices are host mirrors of the
// device slots, like the particle slices: written through, they are uploaded before the next
// device phase; read after a phase, they are downloaded fresh.  The device solver and bond
// storage are created by setupBonds(); bond slices written before it are replaced by the
// bonds it finds (the reference's examples write their initial zeros and -1 there).
// sliceBondFn*() are host-only: the reference never writes its bond_fn_* arrays
// (BondedDEM_Force.hpp:69-71 takes them, no line stores to them).
template <class MemorySpace, int Dimension, int MaxBonds>
class ParticlesBondedDEM : public CabanaDEM::Particles<MemorySpace, Dimension, 1, 0> {
    using Base = CabanaDEM::Particles<MemorySpace, Dimension, 1, 0>;

  public:
    using memory_space = MemorySpace;
    using execution_space = typename MemorySpace::execution_space;
    double delta = 0.0;

    // ParticlesBondedDEM(exec, n) (:49-58); output_folder and bond_params are additions: the
    // folder of output() and the bond model (default: the reference's, every DEM_BQ* bit set,
    // sign-damping 0.1, bond radius = the smaller particle radius)
    template <class ExecSpace>
    ParticlesBondedDEM(const ExecSpace &e, std::size_t n, const std::string &output_folder = "",
                       const dem_bond_params *bond_params = nullptr, std::shared_ptr<Context> ctx = nullptr)
        : Base(e, n, output_folder, ctx) {
        if (bond_params) bp_ = *bond_params;
        else {
            bp_ = dem_bond_params{};
            bp_.quirks = DEM_BOND_REF_COMPAT;
            bp_.beta = 0.1;
            bp_.radius_factor = 1.0;
        }
        for (int f : {DEM_B_IDX, DEM_B_COUNT}) {
            auto m = std::make_shared<Mirror<int>>();
            m->ncomp = f == DEM_B_IDX ? MaxBonds : 1;
            m->data.assign(n * static_cast<size_t>(m->ncomp), f == DEM_B_IDX ? -1 : 0);
            m->fresh = true;
            bi_[f] = m;
        }
        for (int f = DEM_B_INIT_LEN; f <= DEM_B_MT_Z; ++f) {
            if (f == DEM_B_COUNT) continue;
            auto m = std::make_shared<Mirror<double>>();
            m->ncomp = MaxBonds;
            m->data.assign(n * static_cast<size_t>(MaxBonds), 0.0);
            m->fresh = true;
            bd_[f] = m;
        }
        for (auto &m : fn_) {
            m = std::make_shared<Mirror<double>>();
            m->ncomp = MaxBonds;
            m->data.assign(n * static_cast<size_t>(MaxBonds), 0.0);
            m->fresh = true;
        }
    }
    ~ParticlesBondedDEM() {
        if (b_) dem_bonds_destroy(b_);
        if (s_) {
            dem_solver_destroy(s_);
            this->attach_solver(-1);
        }
    }

    void update_mesh_limits(const std::array<double, 3> &lo, const std::array<double, 3> &hi) {
        this->mesh_lo = lo;   // kept for source compatibility: the device grid follows the
        this->mesh_hi = hi;   // particles' bounding box
    }

    // updateParticles(exec, functor) (:60-64): functor(pid) on the host for every particle,
    // then every particle and bond slice written through is uploaded
    template <class ExecSpace, class Functor>
    void updateParticles(const ExecSpace &, const Functor &f) {
        for (int pid = 0; pid < static_cast<int>(this->size()); ++pid) f(pid);
        commit();
    }

    HostSlice<double> sliceBondFnX() { return HostSlice<double>(fn_[0]); }
    HostSlice<double> sliceBondFnY() { return HostSlice<double>(fn_[1]); }
    HostSlice<double> sliceBondFnZ() { return HostSlice<double>(fn_[2]); }
    HostSlice<double> sliceBondFtX() { return bslice_d(DEM_B_FT_X); }
    HostSlice<double> sliceBondFtY() { return bslice_d(DEM_B_FT_Y); }
    HostSlice<double> sliceBondFtZ() { return bslice_d(DEM_B_FT_Z); }
    HostSlice<double> sliceBondMnX() { return bslice_d(DEM_B_MN_X); }
    HostSlice<double> sliceBondMnY() { return bslice_d(DEM_B_MN_Y); }
    HostSlice<double> sliceBondMnZ() { return bslice_d(DEM_B_MN_Z); }
    HostSlice<double> sliceBondMtX() { return bslice_d(DEM_B_MT_X); }
    HostSlice<double> sliceBondMtY() { return bslice_d(DEM_B_MT_Y); }
    HostSlice<double> sliceBondMtZ() { return bslice_d(DEM_B_MT_Z); }
    HostSlice<double> sliceBondInitLen() { return bslice_d(DEM_B_INIT_LEN); }
    HostSlice<int> sliceBondIdx() { return bslice_i(DEM_B_IDX); }
    HostSlice<int> sliceTotalNoBonds() { return bslice_i(DEM_B_COUNT); }

    // setupBonds<ExecSpace>() (:86-171): bond every j with rij < 3 rad(i) among the particles
    // within 4 rad(0), as the reference hard-codes (:130, :152-154); the arguments allow others
    template <class ExecSpace>
    void setupBonds(double factor = 3.0, double search_cutoff = 0.0) {
        this->commit();
        if (!s_) create_device();
        if (!(search_cutoff > 0.0)) search_cutoff = 4.0 * this->sliceRadius().get(0);
        this->context().check(dem_bonds_setup(b_, factor, search_cutoff), "dem_bonds_setup");
        for (auto &kv : bi_) kv.second->dirty = kv.second->fresh = false;
        for (auto &kv : bd_) kv.second->dirty = kv.second->fresh = false;
        this->invalidate();
    }

    // host edits -> device, for every particle and bond slice written since the last phase
    void commit() {
        Base::commit();
        if (!b_) return;
        for (auto &kv : bi_)
            if (kv.second->dirty) {
                this->context().check(dem_bonds_set(b_, kv.first, kv.second->data.data(), (long)kv.second->data.size()),
                                      "dem_bonds_set");
                kv.second->dirty = false;
            }
        for (auto &kv : bd_)
            if (kv.second->dirty) {
                this->context().check(dem_bonds_set(b_, kv.first, kv.second->data.data(), (long)kv.second->data.size()),
                                      "dem_bonds_set");
                kv.second->dirty = false;
            }
    }
    // device -> mirrors on their next read
    void invalidate() {
        Base::invalidate();
        for (auto &kv : bi_) kv.second->fresh = false;
        for (auto &kv : bd_) kv.second->fresh = false;
    }

    // One device phase: slice edits uploaded first, slices stale afterwards.
    template <class F>
    int phase(F &&f, const char *what, int allow = 0) {
        if (!s_) throw Error(std::string(what) + ": call setupBonds first");
        commit();
        const int st = f();
        invalidate();
        this->context().check(st, what, allow);
        return st;
    }
    // The hooks of the reference example, on the device: F += the external force set with
    // setExternalForce (applyTensileForce, tst_01_BDEM:70-117), and gravity then the fix
    // flags set with setFixFlags (applyBoundaryConditions, :19-67).
    void addExternalForce() {
        phase([&] { return dem_apply_external_force(s_); }, "dem_apply_external_force");
    }
    void applyFixFlags() {
        phase([&] { return dem_apply_boundary_conditions(s_); }, "dem_apply_boundary_conditions");
    }
    // The whole bonded loop fused on the device, n steps of dt (dem_bonded_run).
    void run_steps(int n, double dt) {
        set_timestep(dt);
        phase([&] { return dem_bonded_run(b_, n); }, "dem_bonded_run");
    }
    long broken() {
        long c = 0;
        this->context().check(dem_bonds_broken(b_, &c), "dem_bonds_broken");
        return c;
    }
    void set_timestep(double dt) {
        if (!s_) throw Error("set_timestep: call setupBonds first");
        if (dt != dt_) {
            this->context().check(dem_solver_set_timestep(s_, dt), "dem_solver_set_timestep");
            dt_ = dt;
        }
    }
    dem_solver *solver_handle() { return s_; }
    dem_bonds *bonds_handle() { return b_; }

  private:
    void create_device() {
        dem_solver_params sp{};
        sp.dt = dt_;
        const dem_force_params fp{1.0, 1.0, 0.0, 0.0, DEM_REF_COMPAT};
        this->context().check(dem_solver_create(this->context().handle(), this->handle(), nullptr, &fp, &sp, &s_),
                              "dem_solver_create");
        this->attach_solver(1);
        this->context().check(dem_bonds_create(s_, MaxBonds, &bp_, &b_), "dem_bonds_create");
    }
    HostSlice<double> bslice_d(int field) {
        auto &m = bd_[field];
        if (b_ && !m->fresh && !m->dirty) {
            this->context().check(dem_bonds_get(b_, field, m->data.data(), (long)m->data.size()), "dem_bonds_get");
            m->fresh = true;
        }
        return HostSlice<double>(m);
    }
    HostSlice<int> bslice_i(int field) {
        auto &m = bi_[field];
        if (b_ && !m->fresh && !m->dirty) {
            this->context().check(dem_bonds_get(b_, field, m->data.data(), (long)m->data.size()), "dem_bonds_get");
            m->fresh = true;
        }
        return HostSlice<int>(m);
    }

    dem_bond_params bp_{};
    dem_solver *s_ = nullptr;
    dem_bonds *b_ = nullptr;
    double dt_ = 1e-4;   // replaced by the integrator's or run_steps' dt
    std::map<int, std::shared_ptr<Mirror<int>>> bi_;
    std::map<int, std::shared_ptr<Mirror<double>>> bd_;
    std::array<std::shared_ptr<Mirror<double>>, 3> fn_;
};

// resetForcesAndTorques<ExecutionSpace>(particles) (BondedDEM_Force.hpp:16-50): F = tau = 0.
template <class ExecutionSpace, class ParticleType>
void resetForcesAndTorques(ParticleType &particles) {
    particles.phase([&] { return dem_bonded_reset(particles.bonds_handle()); }, "dem_bonded_reset");
}

// computeBondedForce<ExecutionSpace>(particles, dt) (BondedDEM_Force.hpp:53-348): F and tau +=
// every bond's force and moment, in slot order, on top of what the phases before it left.
template <class ExecutionSpace, class ParticleType>
void computeBondedForce(ParticleType &particles, double dt) {
    particles.phase([&] { return dem_bonded_force(particles.bonds_handle(), dt); }, "dem_bonded_force");
}

// BondedDEMIntegrator<ExecutionSpace>(dt) (BondedDEM_Integrator.hpp:15-102): velocity-Verlet
// half-kicks and drift of a ParticlesBondedDEM, with the integrator's dt.
template <class ExecutionSpace>
class BondedDEMIntegrator {
  public:
    explicit BondedDEMIntegrator(double dt) : _dt(dt), _half_dt(0.5 * dt) {}
    template <class ParticlesType>
    void stage1(ParticlesType &p) { stage(p, dem_stage1, "dem_stage1"); }
    template <class ParticlesType>
    void stage2(ParticlesType &p) { stage(p, dem_stage2, "dem_stage2"); }
    template <class ParticlesType>
    void stage3(ParticlesType &p) { stage(p, dem_stage3, "dem_stage3"); }

  private:
    template <class ParticlesType>
    void stage(ParticlesType &p, int (*f)(dem_solver *), const char *what) {
        p.set_timestep(_dt);
        p.phase([&] { return f(p.solver_handle()); }, what);
    }
    double _dt, _half_dt;
};

}  // namespace CabanaBondedDEM
