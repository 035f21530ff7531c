// VTK output and restart of colony state (host side of libpcc_gpu.so).
//
// Writes the reference's ASCII UnstructuredGrid files byte for byte:
// vtk::VTKDataLogger (logger/VTK.h:190-473) as driven by vtk::ParticleLogger
// (logger/ParticleLogger.cpp:13-76), vtk::SimulationLogger
// (logger/SimulationLogger.cpp:9-36) and vtk::ParameterLogger
// (logger/ParameterLogger.cpp:11-40), at one rank: data/<prefix>_<7-digit
// index>_rank_0000.vtu plus <prefix>_<index>.pvtu.  Numbers are formatted as
// an std::ostream with default flags formats them (printf "%g", 6 significant
// digits); points are rounded to float first, as VTKPoints stores them.
//
// The device path snapshots the cell arrays into a second device copy on the
// context's stream (a few tens of microseconds at R = 260), copies that to
// pinned host memory on a side stream, and formats and writes the files on a
// background thread, one thread per data array, so the colony keeps stepping
// while a snapshot is written.
//
// The reader restates vtk::VTKStateLoader (loader/VTKStateLoader.cpp:24-357):
// latest simulation_NNNNNNN.pvtu, its field data, and the particles of the
// same index, with the loader's parsing rules (including that a field value is
// read as the first run of digits, '.' and '-' on its line).
#include <cuda_runtime.h>

#include <sys/stat.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <charconv>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <regex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include <dirent.h>

#include "pcc_kernels.hpp"

namespace pcc {
namespace vtkio {

// ------------------------------------------------------------------ formatting
inline void put_g(std::string& o, double v) {
  char b[40];
  const int k = std::snprintf(b, sizeof b, "%g", v);
  o.append(b, (size_t)k);
}
inline void put_i(std::string& o, long long v) {
  char b[24];
  auto r = std::to_chars(b, b + sizeof b, v);
  o.append(b, (size_t)(r.ptr - b));
}
inline void put_u(std::string& o, unsigned long long v) {
  char b[24];
  auto r = std::to_chars(b, b + sizeof b, v);
  o.append(b, (size_t)(r.ptr - b));
}

// One DataArray of point data: its XML attributes and its formatted body.
struct Array {
  std::string type, name;
  int comps = 1;
  std::string body;  // text between the indent and the newline
};

// Scalar arrays print all values on one line; tuple arrays one tuple per line
// (VTKTypedDataArray::GetDataAsString and its std::array specialisation).
template <class F>
Array scalar_array(const char* type, const char* name, size_t n, F value) {
  Array a;
  a.type = type;
  a.name = name;
  a.comps = 1;
  a.body.reserve(n * 12);
  for (size_t i = 0; i < n; ++i) {
    if (i) a.body += ' ';
    value(a.body, i);
  }
  return a;
}

template <class F>
Array tuple_array(const char* type, const char* name, int comps, size_t n, F tuple) {
  Array a;
  a.type = type;
  a.name = name;
  a.comps = comps;
  a.body.reserve(n * (size_t)comps * 12);
  for (size_t i = 0; i < n; ++i) {
    if (i) a.body += "\n          ";
    tuple(a.body, i);
  }
  return a;
}

// Host copy of the per-cell fields a particle file needs (SoA, gid order).
struct Snapshot {
  size_t n = 0;
  std::vector<double> x, y, z, q0, q1, q2, q3, len, diam, ldot, imp, stress, force, vel;
  std::vector<int> age, ncons;
  void resize(size_t m) {
    n = m;
    for (auto* v : {&x, &y, &z, &q0, &q1, &q2, &q3, &len, &diam, &ldot, &imp, &stress}) v->resize(m);
    force.resize(6 * m);
    vel.resize(6 * m);
    age.resize(m);
    ncons.resize(m);
  }
};

// Unit axis of a cell: utils::Quaternion::getDirectionVector (util/Quaternion.cpp:7-38),
// the quaternion applied to (1, 0, 0), in the same operation order.
inline void axis(double w, double x, double y, double z, double t[3]) {
  const double vx = 1.0, vy = 0.0, vz = 0.0;
  const double c1x = y * vz - z * vy, c1y = z * vx - x * vz, c1z = x * vy - y * vx;
  const double c2x = y * c1z - z * c1y, c2y = z * c1x - x * c1z, c2z = x * c1y - y * c1x;
  const double w2 = 2.0 * w;
  t[0] = vx + w2 * c1x + 2.0 * c2x;
  t[1] = vy + w2 * c1y + 2.0 * c2y;
  t[2] = vz + w2 * c1z + 2.0 * c2z;
}

// The fourteen point-data arrays of ParticleLogger::log, in its order.
std::vector<Array> particle_arrays(const Snapshot& s, const std::vector<size_t>* pick, int rank, bool ghost_copy) {
  const size_t n = pick ? pick->size() : s.n;
  auto at = [&](size_t i) { return pick ? (*pick)[i] : i; };
  std::vector<std::function<Array()>> jobs = {
      [&] { return scalar_array("Int32", "gid", n, [&](std::string& o, size_t i) { put_i(o, (long long)at(i)); }); },
      [&] {
        return tuple_array("Float64", "quaternion", 4, n, [&](std::string& o, size_t i) {
          const size_t k = at(i);
          put_g(o, s.q0[k]);
          o += ' ';
          put_g(o, s.q1[k]);
          o += ' ';
          put_g(o, s.q2[k]);
          o += ' ';
          put_g(o, s.q3[k]);
        });
      },
      [&] {
        return tuple_array("Float64", "orientation", 3, n, [&](std::string& o, size_t i) {
          const size_t k = at(i);
          double t[3];
          axis(s.q0[k], s.q1[k], s.q2[k], s.q3[k], t);
          put_g(o, t[0]);
          o += ' ';
          put_g(o, t[1]);
          o += ' ';
          put_g(o, t[2]);
        });
      },
      [&] {
        return scalar_array("Float64", "orientation_angle", n, [&](std::string& o, size_t i) {
          const size_t k = at(i);
          double t[3];
          axis(s.q0[k], s.q1[k], s.q2[k], s.q3[k], t);
          double a = std::atan2(t[1], t[0]);
          if (a < 0) a += M_PI;
          put_g(o, a);
        });
      },
      [&] {
        return tuple_array("Float64", "lengths", 3, n, [&](std::string& o, size_t i) {
          const size_t k = at(i);
          put_g(o, s.len[k]);
          o += ' ';
          put_g(o, s.diam[k]);
          o += ' ';
          put_g(o, s.diam[k]);
        });
      },
      [&] {
        return scalar_array("Float64", "impedance", n,
                            [&](std::string& o, size_t i) { put_g(o, ghost_copy ? 0.0 : s.imp[at(i)]); });
      },
      [&] { return scalar_array("Float64", "ldot", n, [&](std::string& o, size_t i) { put_g(o, s.ldot[at(i)]); }); },
      [&] {
        return scalar_array("Float64", "stress", n,
                            [&](std::string& o, size_t i) { put_g(o, ghost_copy ? 0.0 : s.stress[at(i)]); });
      },
      [&] {
        return scalar_array("Int32", "number_of_constraints", n,
                            [&](std::string& o, size_t i) { put_i(o, ghost_copy ? 0 : s.ncons[at(i)]); });
      },
      [&] { return scalar_array("Int32", "age", n, [&](std::string& o, size_t i) { put_i(o, s.age[at(i)]); }); },
      [&] {
        return tuple_array("Float64", "forces", 3, n, [&](std::string& o, size_t i) {
          const size_t k = at(i);
          for (int d = 0; d < 3; ++d) {
            if (d) o += ' ';
            put_g(o, ghost_copy ? 0.0 : s.force[6 * k + d]);
          }
        });
      },
      [&] {
        return tuple_array("Float64", "velocity_linear", 3, n, [&](std::string& o, size_t i) {
          const size_t k = at(i);
          for (int d = 0; d < 3; ++d) {
            if (d) o += ' ';
            put_g(o, ghost_copy ? 0.0 : s.vel[6 * k + d]);
          }
        });
      },
      [&] {
        return tuple_array("Float64", "velocity_angular", 3, n, [&](std::string& o, size_t i) {
          const size_t k = at(i);
          for (int d = 0; d < 3; ++d) {
            if (d) o += ' ';
            put_g(o, ghost_copy ? 0.0 : s.vel[6 * k + 3 + d]);
          }
        });
      },
      [&] { return scalar_array("Int32", "rank", n, [&](std::string& o, size_t) { put_i(o, rank); }); },
  };
  std::vector<Array> out(jobs.size());
  // one thread per array: formatting 3e5 cells is ~1 s of snprintf serially
  const bool par = n > 20000;
  std::vector<std::thread> th;
  for (size_t j = 0; j < jobs.size(); ++j) {
    if (par)
      th.emplace_back([&, j] { out[j] = jobs[j](); });
    else
      out[j] = jobs[j]();
  }
  for (auto& t : th) t.join();
  return out;
}

std::string points_body(const Snapshot& s, const std::vector<size_t>* pick) {
  const size_t n = pick ? pick->size() : s.n;
  std::string o;
  o.reserve(n * 40);
  for (size_t i = 0; i < n; ++i) {
    const size_t k = pick ? (*pick)[i] : i;
    o += "          ";
    put_g(o, (double)(float)s.x[k]);
    o += ' ';
    put_g(o, (double)(float)s.y[k]);
    o += ' ';
    put_g(o, (double)(float)s.z[k]);
    o += '\n';
  }
  return o;
}

struct Field {
  std::string type, name, value;
};

bool make_dirs(const std::string& dir) {
  std::string cur;
  size_t i = 0;
  while (i <= dir.size()) {
    size_t j = dir.find('/', i);
    if (j == std::string::npos) j = dir.size();
    cur = dir.substr(0, j);
    if (!cur.empty()) {
      if (mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) return false;
    }
    i = j + 1;
  }
  return true;
}

std::string step_base(const std::string& prefix, unsigned long long index) {
  char b[32];
  std::snprintf(b, sizeof b, "_%07llu", index);
  return prefix + b;
}

// VTKDataLogger::write at one rank (logger/VTK.h:268-304, 308-351, 353-473).
bool write_files(const std::string& outdir, const std::string& prefix, unsigned long long index,
                 const std::vector<Field>& fields, const std::string& points, size_t npoints,
                 const std::vector<Array>& arrays) {
  if (!make_dirs(outdir + "/data")) return false;
  const std::string base = step_base(prefix, index);
  const std::string vtu = outdir + "/data/" + base + "_rank_0000.vtu";
  {
    std::string o;
    o.reserve(points.size() + 64 * 1024);
    o += "<?xml version=\"1.0\"?>\n";
    o += "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
    o += "  <UnstructuredGrid>\n";
    if (!fields.empty()) {
      o += "    <FieldData>\n";
      for (const auto& f : fields) {
        o += "      <DataArray type=\"" + f.type + "\" Name=\"" + f.name +
             "\" NumberOfTuples=\"1\" format=\"ascii\">\n";
        o += "        " + f.value + "\n";
        o += "      </DataArray>\n";
      }
      o += "    </FieldData>\n";
    }
    o += "    <Piece NumberOfPoints=\"";
    put_u(o, npoints);
    o += "\" NumberOfCells=\"0\">\n";
    o += "      <Points>\n";
    o += "        <DataArray type=\"Float32\" Name=\"Points\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    o += points;
    o += "        </DataArray>\n";
    o += "      </Points>\n";
    o += "      <Cells>\n";
    o += "        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n";
    o += "        </DataArray>\n";
    o += "        <DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n";
    o += "        </DataArray>\n";
    o += "        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
    o += "        </DataArray>\n";
    o += "      </Cells>\n";
    FILE* fp = std::fopen(vtu.c_str(), "wb");
    if (!fp) return false;
    bool ok = std::fwrite(o.data(), 1, o.size(), fp) == o.size();
    if (!arrays.empty()) {
      std::string h = "      <PointData>\n";
      ok = ok && std::fwrite(h.data(), 1, h.size(), fp) == h.size();
      for (const auto& a : arrays) {
        std::string head = "        <DataArray type=\"" + a.type + "\" Name=\"" + a.name +
                           "\" NumberOfComponents=\"" + std::to_string(a.comps) + "\" format=\"ascii\">\n          ";
        ok = ok && std::fwrite(head.data(), 1, head.size(), fp) == head.size();
        ok = ok && std::fwrite(a.body.data(), 1, a.body.size(), fp) == a.body.size();
        const char* tail = "\n        </DataArray>\n";
        ok = ok && std::fwrite(tail, 1, std::strlen(tail), fp) == std::strlen(tail);
      }
      h = "      </PointData>\n";
      ok = ok && std::fwrite(h.data(), 1, h.size(), fp) == h.size();
    }
    const char* end = "    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n";
    ok = ok && std::fwrite(end, 1, std::strlen(end), fp) == std::strlen(end);
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) return false;
  }
  std::string p;
  p += "<?xml version=\"1.0\"?>\n";
  p += "<VTKFile type=\"PUnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
  p += "  <PUnstructuredGrid GhostLevel=\"0\">\n";
  if (!fields.empty()) {
    p += "    <PFieldData>\n";
    for (const auto& f : fields)
      p += "      <PDataArray type=\"" + f.type + "\" Name=\"" + f.name + "\" NumberOfComponents=\"1\"/>\n";
    p += "    </PFieldData>\n";
  }
  if (!arrays.empty()) {
    p += "    <PPointData>\n";
    for (const auto& a : arrays)
      p += "      <PDataArray type=\"" + a.type + "\" Name=\"" + a.name + "\" NumberOfComponents=\"" +
           std::to_string(a.comps) + "\"/>\n";
    p += "    </PPointData>\n";
  }
  p += "    <PPoints>\n";
  p += "      <PDataArray type=\"Float32\" Name=\"Points\" NumberOfComponents=\"3\"/>\n";
  p += "    </PPoints>\n";
  p += "    <Piece Source=\"data/" + base + "_rank_0000.vtu\"/>\n";
  p += "  </PUnstructuredGrid>\n";
  p += "</VTKFile>\n";
  FILE* fp = std::fopen((outdir + "/" + base + ".pvtu").c_str(), "wb");
  if (!fp) return false;
  bool ok = std::fwrite(p.data(), 1, p.size(), fp) == p.size();
  return (std::fclose(fp) == 0) && ok;
}

Field fd(const char* name, double v) {
  Field f{"Float64", name, ""};
  put_g(f.value, v);
  return f;
}
Field fi(const char* name, long long v) {
  Field f{"Int32", name, ""};
  put_i(f.value, v);
  return f;
}
Field fu(const char* name, unsigned long long v) {
  Field f{"UInt64", name, ""};
  put_u(f.value, v);
  return f;
}

std::vector<Field> simulation_fields(const pcc_sim_record& r) {
  return {fd("simulation_time_s", r.simulation_time_s), fd("time_since_last_log_s", r.time_since_last_log_s),
          fu("step", r.step),
          fi("num_particles", r.num_particles),
          fu("num_constraints", r.num_constraints),
          fd("colony_radius", r.colony_radius),
          fi("recursive_iterations", r.recursive_iterations),
          fu("bbpgd_iterations", r.bbpgd_iterations),
          fd("max_overlap", r.max_overlap),
          fd("residual", r.residual),
          fd("memory_usage_mb", r.memory_usage_mb),
          fd("peak_memory_mb", r.peak_memory_mb),
          fd("cpu_time_s", r.cpu_time_s),
          fd("mpi_comm_time_s", r.mpi_comm_time_s),
          fd("load_imbalance", r.load_imbalance),
          fd("dt_s", r.dt_s)};
}

// Self-ghost copies at one rank: the cells Domain::exchangeGhostParticles
// copies across the angle-0 boundary of the single sector
// (spatial/Domain.cpp:263-290, 339-403), with the host's libm.
std::vector<size_t> ghost_cells(const Snapshot& s) {
  std::vector<size_t> g;
  for (size_t i = 0; i < s.n; ++i) {
    const double x = s.x[i], y = s.y[i];
    double ang = std::atan2(y, x) * 180.0 / M_PI;
    if (ang < 0) ang += 360.0;
    const double radius = std::sqrt(x * x + y * y);
    if (radius < 8.0) continue;
    double dmin = ang - 0.0, dmax = 360.0 - ang;
    while (dmin > 180.0) dmin -= 360.0;
    while (dmin < -180.0) dmin += 360.0;
    while (dmax > 180.0) dmax -= 360.0;
    while (dmax < -180.0) dmax += 360.0;
    double dist = 0.0;
    if (!(dmin >= 0 && dmax >= 0)) {
      const double m = std::fabs(dmin) < std::fabs(dmax) ? std::fabs(dmin) : std::fabs(dmax);
      dist = radius * std::sin(m * M_PI / 180.0);
    }
    if (dist < 2.5) g.push_back(i);
  }
  return g;
}

bool write_particles(const std::string& outdir, const std::string& prefix, unsigned long long index,
                     const Snapshot& s, const std::vector<size_t>* pick, bool ghost_copy) {
  const auto arrays = particle_arrays(s, pick, 0, ghost_copy);
  return write_files(outdir, prefix, index, {}, points_body(s, pick), pick ? pick->size() : s.n, arrays);
}

void snapshot_from_cells(const pcc_cells* c, size_t n, Snapshot* s) {
  s->resize(n);
  auto cp = [&](std::vector<double>& dst, const double* src) {
    if (src) std::memcpy(dst.data(), src, n * sizeof(double));
    else std::fill(dst.begin(), dst.end(), 0.0);
  };
  cp(s->x, c->x);
  cp(s->y, c->y);
  cp(s->z, c->z);
  cp(s->q0, c->q0);
  cp(s->q1, c->q1);
  cp(s->q2, c->q2);
  cp(s->q3, c->q3);
  cp(s->len, c->length);
  cp(s->diam, c->diameter);
  cp(s->ldot, c->ldot);
  cp(s->imp, c->impedance);
  cp(s->stress, c->stress);
  if (c->force) std::memcpy(s->force.data(), c->force, 6 * n * sizeof(double));
  else std::fill(s->force.begin(), s->force.end(), 0.0);
  if (c->velocity) std::memcpy(s->vel.data(), c->velocity, 6 * n * sizeof(double));
  else std::fill(s->vel.begin(), s->vel.end(), 0.0);
  if (c->age) std::memcpy(s->age.data(), c->age, n * sizeof(int));
  else std::fill(s->age.begin(), s->age.end(), 1);
  if (c->num_constraints) std::memcpy(s->ncons.data(), c->num_constraints, n * sizeof(int));
  else std::fill(s->ncons.begin(), s->ncons.end(), 0);
}

// ------------------------------------------------------------------ reader
struct ArrayData {
  std::string type;
  int comps = 1;
  std::vector<double> v;
};

bool read_lines(const std::string& path, std::vector<std::string>* lines) {
  std::ifstream f(path);
  if (!f.is_open()) return false;
  std::string l;
  while (std::getline(f, l)) lines->push_back(l);
  return true;
}

std::string attr(const std::string& tag, const char* key) {
  const std::string k = std::string(key) + "=\"";
  size_t a = tag.find(k);
  if (a == std::string::npos) return "";
  a += k.size();
  size_t b = tag.find('"', a);
  return b == std::string::npos ? "" : tag.substr(a, b - a);
}

// VTKStateLoader::readVTUFile (VTKStateLoader.cpp:217-301).
bool read_vtu(const std::string& path, std::map<std::string, ArrayData>* out, std::string* err) {
  std::vector<std::string> lines;
  if (!read_lines(path, &lines)) {
    *err = "Could not open VTU file: " + path;
    return false;
  }
  static const std::regex open_tag("<DataArray\\s+[^>]*>");
  bool reading = false;
  std::string name;
  ArrayData cur;
  std::string buf;
  for (const auto& line : lines) {
    if (line.rfind("line:", 0) == 0) continue;
    if (!reading) {
      std::smatch m;
      if (std::regex_search(line, m, open_tag)) {
        const std::string tag = m[0].str();
        name = attr(tag, "Name");
        cur = ArrayData();
        cur.type = attr(tag, "type");
        const std::string c = attr(tag, "NumberOfComponents");
        cur.comps = c.empty() ? 1 : std::stoi(c);
        reading = true;
        buf.clear();
      }
    } else if (line.find("</DataArray>") != std::string::npos) {
      if (!name.empty()) {
        const char* p = buf.data();
        const char* e = p + buf.size();
        while (p < e) {
          while (p < e && std::isspace((unsigned char)*p)) ++p;
          const char* q = p;
          while (q < e && !std::isspace((unsigned char)*q)) ++q;
          if (q > p) {
            double v;
            auto r = std::from_chars(p, q, v);
            if (r.ec != std::errc() || r.ptr != q) {
              *err = "Conversion error";
              return false;
            }
            cur.v.push_back(v);
          }
          p = q;
        }
        (*out)[name] = cur;
      }
      reading = false;
      name.clear();
    } else {
      buf += line;
      buf += ' ';
    }
  }
  return true;
}

}  // namespace vtkio

void vtk_clear_prefix(const std::string& dir, const std::string& prefix) {
  for (const std::string sub : {std::string(""), std::string("/data")}) {
    const std::string d = dir + sub;
    const char* ext = sub.empty() ? ".pvtu" : ".vtu";
    const size_t el = std::strlen(ext);
    if (DIR* dp = opendir(d.c_str())) {
      std::vector<std::string> gone;
      while (dirent* de = readdir(dp)) {
        const std::string f = de->d_name;
        if (f.size() > el && f.compare(f.size() - el, el, ext) == 0 && f.rfind(prefix, 0) == 0) gone.push_back(f);
      }
      closedir(dp);
      for (const auto& f : gone) std::remove((d + "/" + f).c_str());
    }
  }
}

bool vtk_write_trace(const std::string& dir, unsigned long long first_index,
                     const std::vector<pcc_bbpgd_trace_step>& steps) {
  using namespace vtkio;
  unsigned long long index = first_index;
  for (const auto& t : steps) {
    // BBPGDLogger::log (logger/BBPGDLogger.cpp:12-27): one file pair per record
    const std::vector<Field> f = {fu("step", t.step),
                                  fu("recursive_iteration", t.recursive_iteration),
                                  fu("total_constraints", t.total_constraints),
                                  fd("residual", t.residual),
                                  fd("step_size", t.step_size),
                                  fd("linear", t.linear),
                                  fd("quadratic", t.quadratic),
                                  fd("growth", t.growth),
                                  fd("total", t.total)};
    if (!write_files(dir, "bbpgdtrace", index++, f, "", 0, {})) return false;
  }
  return true;
}

}  // namespace pcc

using namespace pcc;
using namespace pcc::vtkio;

struct pcc_vtk_writer_state {
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::function<bool()>> work;
  std::thread th;
  bool stop = false;
  int failed = 0;
  size_t pending = 0;
  std::string err;
};

namespace {

void writer_loop(pcc_vtk_writer_state* w) {
  for (;;) {
    std::function<bool()> job;
    {
      std::unique_lock<std::mutex> l(w->mu);
      w->cv.wait(l, [&] { return w->stop || !w->work.empty(); });
      if (w->work.empty()) return;
      job = std::move(w->work.front());
      w->work.pop_front();
    }
    const bool ok = job();
    {
      std::lock_guard<std::mutex> l(w->mu);
      if (!ok) w->failed++;
      w->pending--;
    }
    w->cv.notify_all();
  }
}

}  // namespace

namespace pcc {
void vtk_writer_shutdown(pcc_ctx* ctx) {
  pcc_vtk_writer_state* w = ctx->vtk_writer;
  if (!w) return;
  {
    std::lock_guard<std::mutex> l(w->mu);
    w->stop = true;
  }
  w->cv.notify_all();
  if (w->th.joinable()) w->th.join();
  delete w;
  ctx->vtk_writer = nullptr;
}
}  // namespace pcc

extern "C" {

pcc_status pcc_vtk_write_particles(const char* outdir, const char* prefix, unsigned long long index,
                                   const pcc_cells* cells, size_t n, int ghost_copies) {
  if (!outdir || !prefix || (n && !cells)) return PCC_ERR_INVALID;
  Snapshot s;
  if (n) snapshot_from_cells(cells, n, &s);
  if (ghost_copies) {
    const auto pick = ghost_cells(s);
    return write_particles(outdir, prefix, index, s, &pick, true) ? PCC_OK : PCC_ERR_INVALID;
  }
  return write_particles(outdir, prefix, index, s, nullptr, false) ? PCC_OK : PCC_ERR_INVALID;
}

pcc_status pcc_vtk_write_simulation(const char* outdir, unsigned long long index, const pcc_sim_record* rec) {
  if (!outdir || !rec) return PCC_ERR_INVALID;
  return write_files(outdir, "simulation", index, simulation_fields(*rec), "", 0, {}) ? PCC_OK : PCC_ERR_INVALID;
}

pcc_status pcc_vtk_write_trace(const char* outdir, unsigned long long first_index, const pcc_bbpgd_trace_step* steps,
                               size_t n) {
  if (!outdir || (n && !steps)) return PCC_ERR_INVALID;
  return vtk_write_trace(outdir, first_index, std::vector<pcc_bbpgd_trace_step>(steps, steps + n)) ? PCC_OK
                                                                                                  : PCC_ERR_INVALID;
}

pcc_status pcc_vtk_write_parameters(const char* outdir, unsigned long long index, const pcc_params* p) {
  if (!outdir || !p) return PCC_ERR_INVALID;
  // ParameterLogger::log (logger/ParameterLogger.cpp:11-40); the three
  // settings the device path has no use for carry the reference CLI defaults
  // (util/CLIParser.h:165-195): growth_factor 1.5, particle_preallocation_factor
  // 20; min_box_size is (l0 + 1, l0 + 1, 0) as the parser sets it (233-236).
  std::vector<Field> f = {fd("dt_s", p->dt),
                          fd("end_radius", p->end_radius),
                          fd("log_every_colony_radius_delta", p->log_every_colony_radius_delta),
                          fd("log_every_sim_time_delta", p->log_every_sim_time_delta),
                          fd("min_box_size_x", p->l0 + 1.0),
                          fd("min_box_size_y", p->l0 + 1.0),
                          fd("min_box_size_z", 0.0),
                          fd("xi", p->xi),
                          fd("TAU", p->tau),
                          fd("l0", p->l0),
                          fd("LAMBDA", p->lambda),
                          fd("temperature", p->temperature),
                          fd("kcc", p->kcc),
                          fu("max_bbpgd_iterations", (unsigned long long)p->max_bbpgd_iterations),
                          fu("max_recursive_iterations", (unsigned long long)p->max_recursive_iterations),
                          fd("linked_cell_size", p->linked_cell_size),
                          fd("growth_factor", 1.5),
                          fd("particle_preallocation_factor", 20.0),
                          fi("mode", p->mode == PCC_MODE_HARD ? 0 : 1)};
  return write_files(outdir, "parameters", index, f, "", 0, {}) ? PCC_OK : PCC_ERR_INVALID;
}

pcc_status pcc_log_vtk(pcc_ctx* ctx, const char* outdir, unsigned long long index, const pcc_sim_record* rec) {
  if (!ctx || !outdir) return PCC_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaStream_t s = ctx->stream;
  const size_t n = ctx->n;
  cudaError_t e;
  if (!ctx->vtk_writer) {
    ctx->vtk_writer = new pcc_vtk_writer_state();
    ctx->vtk_writer->th = std::thread(writer_loop, ctx->vtk_writer);
  }
  if (!ctx->vtk_stream) {
    if ((e = cudaStreamCreateWithFlags(&ctx->vtk_stream, cudaStreamNonBlocking))) return PCC_ERR_CUDA;
    if ((e = cudaEventCreateWithFlags(&ctx->vtk_ev, cudaEventDisableTiming))) return PCC_ERR_CUDA;
  }
  // device-side copy on the colony's stream (ordered after the last step),
  // then the host copy on the side stream while the colony steps on
  auto snap = std::make_shared<Snapshot>();
  snap->resize(n);
  const size_t nd = 12 * n + 12 * n;  // 12 scalars + force + velocity
  if ((e = ctx->vtk_dev.reserve(nd + 1, 0, s))) return PCC_ERR_CUDA;
  if ((e = ctx->vtk_idev.reserve(2 * n + 1, 0, s))) return PCC_ERR_CUDA;
  CellsView v = ctx->cells.view();
  const double* src[12] = {v.x, v.y, v.z, v.q0, v.q1, v.q2, v.q3, v.len, v.diam, v.ldot, v.imp, v.stress};
  double* d = ctx->vtk_dev.p;
  if (n) {
    for (int k = 0; k < 12; ++k) cudaMemcpyAsync(d + k * n, src[k], n * sizeof(double), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(d + 12 * n, v.force, 6 * n * sizeof(double), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(d + 18 * n, v.vel, 6 * n * sizeof(double), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(ctx->vtk_idev.p, v.age, n * sizeof(int), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(ctx->vtk_idev.p + n, v.ncons, n * sizeof(int), cudaMemcpyDeviceToDevice, s);
  }
  cudaEventRecord(ctx->vtk_ev, s);
  cudaStreamWaitEvent(ctx->vtk_stream, ctx->vtk_ev, 0);
  // pinned staging owned by the job (freed by the writer thread)
  double* hd = nullptr;
  int* hi = nullptr;
  if (n) {
    if ((e = cudaMallocHost(&hd, nd * sizeof(double)))) return PCC_ERR_NOMEM;
    if ((e = cudaMallocHost(&hi, 2 * n * sizeof(int)))) {
      cudaFreeHost(hd);
      return PCC_ERR_NOMEM;
    }
    cudaMemcpyAsync(hd, d, nd * sizeof(double), cudaMemcpyDeviceToHost, ctx->vtk_stream);
    cudaMemcpyAsync(hi, ctx->vtk_idev.p, 2 * n * sizeof(int), cudaMemcpyDeviceToHost, ctx->vtk_stream);
  }
  cudaEvent_t done = nullptr;
  e = cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
  if (!e) e = cudaEventRecord(done, ctx->vtk_stream);
  if (!e) e = cudaGetLastError();
  if (e) {
    cudaStreamSynchronize(ctx->vtk_stream);  // no copy may still target the staging buffers
    if (done) cudaEventDestroy(done);
    if (hd) cudaFreeHost(hd);
    if (hi) cudaFreeHost(hi);
    ctx->err = std::string("pcc_log_vtk: ") + cudaGetErrorString(e);
    return PCC_ERR_CUDA;
  }
  const std::string dir(outdir);
  const bool with_rec = rec != nullptr;
  const pcc_sim_record r = rec ? *rec : pcc_sim_record{};
  const int dev = ctx->device;
  auto job = [snap, hd, hi, n, done, dir, index, with_rec, r, dev]() -> bool {
    cudaSetDevice(dev);
    const bool copied = cudaEventSynchronize(done) == cudaSuccess;
    cudaEventDestroy(done);
    if (copied && n) {
      Snapshot& s = *snap;
      std::vector<double>* dst[12] = {&s.x, &s.y, &s.z, &s.q0, &s.q1, &s.q2, &s.q3, &s.len, &s.diam, &s.ldot, &s.imp,
                                      &s.stress};
      for (int k = 0; k < 12; ++k) std::memcpy(dst[k]->data(), hd + k * n, n * sizeof(double));
      for (size_t i = 0; i < n; ++i) {
        for (int c = 0; c < 6; ++c) {
          s.force[6 * i + c] = hd[12 * n + 6 * i + c];
          s.vel[6 * i + c] = hd[18 * n + 6 * i + c];
        }
      }
      std::memcpy(s.age.data(), hi, n * sizeof(int));
      std::memcpy(s.ncons.data(), hi + n, n * sizeof(int));
    }
    if (hd) cudaFreeHost(hd);
    if (hi) cudaFreeHost(hi);
    if (!copied) return false;
    bool ok = write_particles(dir, "particles", index, *snap, nullptr, false);
    const auto ghosts = ghost_cells(*snap);
    ok = write_particles(dir, "ghost_particles", index, *snap, &ghosts, true) && ok;
    if (with_rec) ok = write_files(dir, "simulation", index, simulation_fields(r), "", 0, {}) && ok;
    return ok;
  };
  {
    std::lock_guard<std::mutex> l(ctx->vtk_writer->mu);
    ctx->vtk_writer->work.push_back(std::move(job));
    ctx->vtk_writer->pending++;
  }
  ctx->vtk_writer->cv.notify_all();
  return PCC_OK;
}

pcc_status pcc_log_vtk_wait(pcc_ctx* ctx) {
  if (!ctx) return PCC_ERR_INVALID;
  pcc_vtk_writer_state* w = ctx->vtk_writer;
  if (!w) return PCC_OK;
  std::unique_lock<std::mutex> l(w->mu);
  w->cv.wait(l, [&] { return w->pending == 0; });
  const int failed = w->failed;
  w->failed = 0;
  if (failed) {
    ctx->err = "pcc_log_vtk: writing a VTK file failed";
    return PCC_ERR_INVALID;
  }
  return PCC_OK;
}

pcc_status pcc_vtk_load(const char* vtk_path, pcc_cells* out, size_t cap, size_t* n, double* sim_time,
                        long long* step, double* dt) {
  if (!vtk_path || !n) return PCC_ERR_INVALID;
  // Domain::initializeFromVTK (spatial/Domain.cpp:650-690): a file path means its directory
  std::string dir(vtk_path);
  struct stat st;
  if (stat(dir.c_str(), &st) != 0) return PCC_ERR_INVALID;
  if (S_ISREG(st.st_mode)) {
    const size_t k = dir.rfind('/');
    dir = k == std::string::npos ? "." : dir.substr(0, k);
  }
  struct stat sd;
  if (stat((dir + "/data").c_str(), &sd) != 0) return PCC_ERR_INVALID;
  // latest simulation_NNNNNNN.pvtu (VTKStateLoader::findLatestTimestep)
  static const std::regex pat("simulation_\\d{7}\\.pvtu");
  long long latest = -1;
  if (DIR* d = opendir(dir.c_str())) {
    while (dirent* de = readdir(d)) {
      const std::string f = de->d_name;
      if (std::regex_match(f, pat)) latest = std::max(latest, std::stoll(f.substr(11, 7)));
    }
    closedir(d);
  }
  if (latest < 0) return PCC_ERR_INVALID;
  char num[24];
  std::snprintf(num, sizeof num, "%07lld", latest);
  // field data of the simulation file's first piece (VTKStateLoader::readFieldData)
  std::vector<std::string> lines;
  if (!read_lines(dir + "/simulation_" + num + ".pvtu", &lines)) return PCC_ERR_INVALID;
  static const std::regex piece("<Piece\\s+Source=\"([^\"]+)\".*>");
  std::string vtu;
  for (const auto& l : lines) {
    std::smatch m;
    if (std::regex_search(l, m, piece)) {
      vtu = dir + "/" + m[1].str();
      break;
    }
  }
  if (vtu.empty()) return PCC_ERR_INVALID;
  std::vector<std::string> vl;
  if (!read_lines(vtu, &vl)) return PCC_ERR_INVALID;
  static const std::regex field("<DataArray.*Name=\"([^\"]+)\".*>");
  static const std::regex value("\\s*([\\d.-]+)\\s*");
  std::map<std::string, double> fields;
  bool reading = false;
  std::string cur;
  for (const auto& l : vl) {
    if (!reading) {
      std::smatch m;
      if (std::regex_search(l, m, field)) {
        cur = m[1].str();
        reading = true;
      }
    } else {
      std::smatch m;
      if (std::regex_search(l, m, value)) {
        try {
          fields[cur] = std::stod(m[1].str());
        } catch (...) {
        }
        reading = false;
      }
    }
    if (l.find("</FieldData>") != std::string::npos) break;
  }
  // particles of the same index, every piece (VTKStateLoader::loadParticles)
  std::vector<std::string> pl;
  if (!read_lines(dir + "/particles_" + num + ".pvtu", &pl)) return PCC_ERR_INVALID;
  static const std::regex src(".*Source=\"([^\"]+)\".*");
  std::vector<double> pos, quat, len, force, vlin, vang;
  for (const auto& l : pl) {
    std::smatch m;
    if (!std::regex_match(l, m, src)) continue;
    std::map<std::string, ArrayData> arrays;
    std::string err;
    if (!read_vtu(dir + "/" + m[1].str(), &arrays, &err)) return PCC_ERR_INVALID;
    const auto& P = arrays["Points"].v;
    const size_t k = P.size() / 3;
    auto need = [&](const char* name, size_t comps) -> const std::vector<double>* {
      const auto& v = arrays[name].v;
      return v.size() >= comps * k ? &v : nullptr;
    };
    const auto *Q = need("quaternion", 4), *L = need("lengths", 3), *F = need("forces", 3),
               *VL = need("velocity_linear", 3), *VA = need("velocity_angular", 3);
    if (!Q || !L || !F || !VL || !VA) return PCC_ERR_INVALID;
    for (size_t i = 0; i < k; ++i) {
      pos.insert(pos.end(), {P[3 * i], P[3 * i + 1], P[3 * i + 2]});
      quat.insert(quat.end(), {(*Q)[4 * i], (*Q)[4 * i + 1], (*Q)[4 * i + 2], (*Q)[4 * i + 3]});
      len.push_back((*L)[3 * i]);
      force.insert(force.end(), {(*F)[3 * i], (*F)[3 * i + 1], (*F)[3 * i + 2]});
      vlin.insert(vlin.end(), {(*VL)[3 * i], (*VL)[3 * i + 1], (*VL)[3 * i + 2]});
      vang.insert(vang.end(), {(*VA)[3 * i], (*VA)[3 * i + 1], (*VA)[3 * i + 2]});
    }
  }
  const size_t m = len.size();
  *n = m;
  if (sim_time) *sim_time = fields["simulation_time_s"];
  if (step) *step = (long long)fields["step"];
  if (dt) *dt = fields["dt_s"];
  if (!out) return PCC_OK;
  if (cap < m) return PCC_ERR_CAPACITY;
  // Particle(gid, position, quaternion, length, l0 = 1, diameter = 0.5):
  // age 1, impedance 0, torque 0; force and both velocities from the file
  for (size_t i = 0; i < m; ++i) {
    if (out->x) out->x[i] = pos[3 * i];
    if (out->y) out->y[i] = pos[3 * i + 1];
    if (out->z) out->z[i] = pos[3 * i + 2];
    if (out->q0) out->q0[i] = quat[4 * i];
    if (out->q1) out->q1[i] = quat[4 * i + 1];
    if (out->q2) out->q2[i] = quat[4 * i + 2];
    if (out->q3) out->q3[i] = quat[4 * i + 3];
    if (out->length) out->length[i] = len[i];
    if (out->l0) out->l0[i] = 1.0;
    if (out->diameter) out->diameter[i] = 0.5;
    if (out->ldot) out->ldot[i] = 0.0;
    if (out->impedance) out->impedance[i] = 0.0;
    if (out->stress) out->stress[i] = 0.0;
    if (out->age) out->age[i] = 1;
    if (out->num_constraints) out->num_constraints[i] = 0;
    if (out->force)
      for (int c = 0; c < 6; ++c) out->force[6 * i + c] = c < 3 ? force[3 * i + c] : 0.0;
    if (out->velocity)
      for (int c = 0; c < 6; ++c) out->velocity[6 * i + c] = c < 3 ? vlin[3 * i + c] : vang[3 * i + c - 3];
  }
  return PCC_OK;
}

pcc_status pcc_set_clock(pcc_ctx* ctx, double sim_time, long long iteration) {
  if (!ctx || iteration < 0) return PCC_ERR_INVALID;
  ctx->sim_time = sim_time;
  ctx->iter = iteration;
  return PCC_OK;
}

}  // extern "C"
