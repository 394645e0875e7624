/*
 * aslb_asl_io.hpp -- ASL's writer, timer, values and parameters manager for
 * programs of the LBGK path: WriterVTKXML (src/writers/aslVTKFormatWriters.h),
 * Timer (src/utilities/aslTimer.h), UValue (src/utilities/aslUValue.h),
 * Parameter / ApplicationParametersManager (src/utilities/
 * aslParametersManager.h) of the reference. Header-only, without VTK or
 * Boost.
 */
#ifndef ASLB_ASL_IO_HPP
#define ASLB_ASL_IO_HPP

#include <cctype>
#include <filesystem>

#include "aslb_asl.hpp"

namespace asl {

// ---- WriterVTKXML -----------------------------------------------------------
//
// Every write() produces <file>_<n>.vti: VTK XML ImageData, appended raw
// binary data, the interior cells of every registered field. As in ASL's
// casts (src/utilities/aslVTKCasters.cxx:166-181) the axes are reversed --
// ASL's arrays are z fastest, VTK's x fastest -- and so are the components
// of vector fields. FP64 fields stay FP64, everything else is FP32.
class WriterVTKXML {
  std::string file_;
  struct Field {
    std::string name;
    const AbstractData* data;
    unsigned int ncomp;
  };
  std::vector<Field> fields_;
  unsigned int numOfWrites_ = 0;

 public:
  explicit WriterVTKXML(const std::string& file) : file_(file) {}
  void addScalars(const std::string& name, AbstractData& d) { fields_.push_back({name, &d, 1}); }
  void addVector(const std::string& name, AbstractData& d) {
    if (d.getEContainerSize() != 3) errorMessage("WriterVTKXML::addVector: a vector field needs 3 components");
    fields_.push_back({name, &d, 3});
  }
  unsigned int getNumOfWrites() const { return numOfWrites_; }
  void write() {
    if (fields_.empty()) errorMessage("WriterVTKXML::write() - there are no fields to write");
    const Block& in = fields_[0].data->getInternalBlock();
    const AVec<int> n = in.getSize();
    std::vector<std::string> blobs;
    std::ostringstream heads;
    size_t off = 0;
    std::string first;
    for (const Field& f : fields_) {
      if (f.data->getInternalBlock().getSize() != n) errorMessage("WriterVTKXML::write: fields of different blocks");
      const std::vector<double>& v = f.data->values();
      const int gh = (int)f.data->getGhostLayer();
      const AVec<int> g = f.data->getBlock().getSize();
      const size_t cells = f.data->cells();
      const bool dbl = f.data->getTypeID() == acl::TYPE_DOUBLE;
      std::string raw;
      for (int x = 0; x < n[0]; ++x)
        for (int y = 0; y < n[1]; ++y)
          for (int z = 0; z < n[2]; ++z) {
            const size_t a = ((size_t)(x + gh) * g[1] + (y + gh)) * g[2] + (z + gh);
            for (int c = (int)f.ncomp - 1; c >= 0; --c) {
              const double val = v[(size_t)c * cells + a];
              if (dbl) {
                raw.append((const char*)&val, sizeof(double));
              } else {
                const float fv = float(val);
                raw.append((const char*)&fv, sizeof(float));
              }
            }
          }
      const uint64_t len = raw.size();
      blobs.push_back(std::string((const char*)&len, sizeof(len)) + raw);
      heads << "        <DataArray type=\"" << (dbl ? "Float64" : "Float32") << "\" Name=\"" << f.name << "\""
            << (f.ncomp == 3 ? " NumberOfComponents=\"3\"" : "") << " format=\"appended\" offset=\"" << off
            << "\"/>\n";
      off += blobs.back().size();
      if (first.empty() && f.ncomp == 1) first = f.name;
    }
    std::ostringstream ext, head;
    ext << "0 " << n[2] - 1 << " 0 " << n[1] - 1 << " 0 " << n[0] - 1;
    head.precision(17);
    head << "<?xml version=\"1.0\"?>\n<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" "
            "header_type=\"UInt64\">\n"
         << "  <ImageData WholeExtent=\"" << ext.str() << "\" Origin=\"" << in.position[2] << " " << in.position[1]
         << " " << in.position[0] << "\" Spacing=\"" << in.dx << " " << in.dx << " " << in.dx << "\">\n"
         << "    <Piece Extent=\"" << ext.str() << "\">\n"
         << "      <PointData" << (first.empty() ? "" : " Scalars=\"" + first + "\"") << ">\n"
         << heads.str() << "      </PointData>\n      <CellData>\n      </CellData>\n    </Piece>\n"
         << "  </ImageData>\n  <AppendedData encoding=\"raw\">\n   _";
    const std::string path = file_ + "_" + std::to_string(numOfWrites_) + ".vti";
    std::ofstream o(path, std::ios::binary);
    if (!o) errorMessage("WriterVTKXML::write: cannot open " + path);
    o << head.str();
    for (const std::string& b : blobs) o.write(b.data(), (std::streamsize)b.size());
    o << "\n  </AppendedData>\n</VTKFile>\n";
    if (!o) errorMessage("WriterVTKXML::write: cannot write " + path);
    ++numOfWrites_;
  }
};

// ---- Timer (src/utilities/aslTimer.h:32-52) ----------------------------------

//
// start() and stop() first wait for the work queued on the device
// (aslb_synchronize), so the timer measures finished steps as ASL's blocking
// launches do; without a device they only read the clocks.
class Timer {
  std::chrono::high_resolution_clock::time_point realTimeMark_;
  std::clock_t processorTimeMark_ = 0;
  std::chrono::duration<double> realTimeElapsed_{0};
  double processorTimeElapsed_ = 0;

 public:
  void start() {
    (void)aslb_synchronize();
    processorTimeMark_ = std::clock();
    realTimeMark_ = std::chrono::high_resolution_clock::now();
  }
  void stop() {
    (void)aslb_synchronize();
    processorTimeElapsed_ += double(std::clock() - processorTimeMark_);
    realTimeElapsed_ += std::chrono::duration_cast<std::chrono::duration<double>>(
        std::chrono::high_resolution_clock::now() - realTimeMark_);
  }
  double realTime() const { return realTimeElapsed_.count(); }
  double processorTime() const { return processorTimeElapsed_ / CLOCKS_PER_SEC; }
  double processorLoad() const { return processorTime() / realTime(); }
  void reset() {
    processorTimeElapsed_ = 0;
    realTimeElapsed_ = std::chrono::duration<double>(0);
  }
  double estimatedDuration(double completeness) const { return realTimeElapsed_.count() / completeness; }
};

// ---- UValue (src/utilities/aslUValue.h:32-52) ---------------------------------

template <typename T>
class UValue {
  std::shared_ptr<T> p_;

 public:
  UValue() : p_(std::make_shared<T>()) {}
  explicit UValue(const T& a) : p_(std::make_shared<T>(a)) {}
  const T& operator=(const T& a) { return (*p_ = a); }
  const T& v() const { return *p_; }
  T& v() { return *p_; }
  std::shared_ptr<T> p() { return p_; }
};
template <typename T> inline bool operator==(const UValue<T>& a, const T& v) { return a.v() == v; }
template <typename T> inline bool operator!=(const UValue<T>& a, const T& v) { return a.v() != v; }

// ---- parameters (src/utilities/aslParametersManager.h:44-196) -----------------
//
// Parameters register with the manager declared before them and are read by
// load(argc, argv) from the command line ("--key value", "--key=value"; a
// vector as "--size '30 20 50'") and from a parameters file given as the
// first free argument ("key = value" lines, '#' comments). --device N
// selects the CUDA device (ASL: --platform / --device select the OpenCL
// device); -h / --help lists the parameters.

namespace aslb_detail {
struct ParamEntry {
  std::string key, description, units;
  bool required;
  std::function<void(const std::string&)> set;
  std::function<std::string()> get;
};
inline std::vector<ParamEntry>& param_registry() {
  static std::vector<ParamEntry> r;
  return r;
}
template <typename T> inline void parse_value(const std::string& s, T& v) {
  std::istringstream is(s);
  if (!(is >> v)) errorMessage("cannot read the value \"" + s + "\"");
}
template <> inline void parse_value<std::string>(const std::string& s, std::string& v) { v = s; }
template <> inline void parse_value<bool>(const std::string& s, bool& v) {
  v = (s == "1" || s == "true" || s == "yes" || s == "on");
}
template <typename T> inline void parse_value(const std::string& s, AVec<T>& v) {
  std::istringstream is(s);
  std::vector<T> xs;
  T x;
  while (is >> x) xs.push_back(x);
  if (xs.empty()) errorMessage("cannot read the vector \"" + s + "\"");
  v = xs;
}
template <typename T> inline std::string show(const T& v) {
  std::ostringstream o;
  o << v;
  return o.str();
}
}  // namespace aslb_detail

template <typename T>
class Parameter {
  UValue<T> parameter;
  std::string key;

  void enlist(bool required, const char* description, const char* units) {
    UValue<T> p = parameter;
    aslb_detail::param_registry().push_back(
        {key, description, units, required, [p](const std::string& s) mutable { aslb_detail::parse_value(s, p.v()); },
         [p]() { return aslb_detail::show(p.v()); }});
  }

 public:
  Parameter(const char* key_, const char* description_, const char* units_ = "") : key(key_) {
    enlist(true, description_, units_);
  }
  Parameter(T defaultValue, const char* key_, const char* description_, const char* units_ = "")
      : parameter(defaultValue), key(key_) {
    enlist(false, description_, units_);
  }
  const T& v() const { return parameter.v(); }
  T& v() { return parameter.v(); }
  std::shared_ptr<T> p() { return parameter.p(); }
};

class ParametersManager {
 protected:
  std::string name_, version_;
  std::string dir_;  // absolute directory of the parameters file, with a trailing '/'

 public:
  ParametersManager() {}
  // the directory of the parameters file given to load(), else the current
  // one (src/utilities/aslParametersManager.cxx:352-355, 487-492)
  std::string getDir() { return dir_; }
  // "key = value" lines
  void loadParametersFile(const std::string& path) {
    std::ifstream in(path);
    if (!in) errorMessage("ParametersManager: cannot open the parameters file " + path);
    std::string line;
    while (std::getline(in, line)) {
      const size_t hash = line.find('#');
      if (hash != std::string::npos) line.resize(hash);
      const size_t eq = line.find('=');
      if (eq == std::string::npos) continue;
      auto trim = [](std::string s) {
        const size_t b = s.find_first_not_of(" \t\r\"");
        const size_t e = s.find_last_not_of(" \t\r\"");
        return b == std::string::npos ? std::string() : s.substr(b, e - b + 1);
      };
      set(trim(line.substr(0, eq)), trim(line.substr(eq + 1)));
    }
  }
  void set(const std::string& key, const std::string& value) {
    for (auto& e : aslb_detail::param_registry())
      if (e.key == key) {
        e.set(value);
        e.required = false;
        return;
      }
    errorMessage("unknown parameter \"" + key + "\"");
  }
};

class ApplicationParametersManager : public ParametersManager {
 public:
  ApplicationParametersManager(const char* applicationName, const char* applicationVersion) {
    name_ = applicationName;
    version_ = applicationVersion;
    aslb_detail::param_registry().clear();
  }
  void load(int argc, char* argv[]) {
    int device = -1;
    std::filesystem::path dir(".");
    for (int i = 1; i < argc; ++i) {
      std::string a = argv[i];
      if (a == "-h" || a == "--help") {
        std::cout << name_ << " " << version_ << "\n  --device N   CUDA device\n";
        for (auto& e : aslb_detail::param_registry())
          std::cout << "  --" << e.key << " (" << (e.required ? "required" : e.get()) << ") " << e.description
                    << (e.units.empty() ? "" : " [" + e.units + "]") << "\n";
        std::exit(0);
      }
      if (a.rfind("--", 0) == 0) {
        std::string key = a.substr(2), value;
        const size_t eq = key.find('=');
        if (eq != std::string::npos) {
          value = key.substr(eq + 1);
          key.resize(eq);
        } else {
          if (i + 1 >= argc) errorMessage("missing value of --" + key);
          value = argv[++i];
        }
        if (key == "device") {
          aslb_detail::parse_value(value, device);
        } else if (key == "platform") {
          // one platform: CUDA
        } else {
          set(key, value);
        }
      } else {
        loadParametersFile(a);
        dir = std::filesystem::path(a).parent_path();
        if (dir.empty()) dir = ".";
      }
    }
    std::error_code ec;
    const std::filesystem::path abs = std::filesystem::canonical(dir, ec);
    dir_ = (ec ? dir : abs).string();
    if (dir_.empty() || dir_.back() != '/') dir_ += '/';
    for (auto& e : aslb_detail::param_registry())
      if (e.required) errorMessage("the parameter \"" + e.key + "\" is required");
    if (device >= 0) aslb_detail::check(aslb_set_device(device), "ApplicationParametersManager: --device");
  }
};

// ---- readSurface (src/readers/aslVTKFormatReaders.h:66-80) -------------------
//
// An STL surface (binary or ASCII) sampled into a map by the library's CUDA
// distance kernels (aslb_read_stl, aslb_surface_map), as ASL's surfaceToData
// samples VTK's implicit modeller (src/readers/aslVTKFormatReaders.cxx:
// 132-216): the unsigned distance d to the nearest triangle (exact within
// four cells of the surface) stored as (d - 1.2 dx) / (1.8 dx) on the given
// block, or as (d - 1.8 dx) / (1.8 dx) on the surface's bounds grown by
// 3.6 dx, or by the given fractions of its extent per face. The sampled grid
// is the container's block with its ghost layer. File coordinates (x, y, z)
// are ASL's (z, y, x). VTK XML PolyData (.vtp) is read by the Python
// library's reader (asl_b200.surface); here it is reported as unsupported.
namespace aslb_detail {
inline std::vector<float> surface_triangles(const std::string& fileName) {
  std::string ext = fileName.size() >= 4 ? fileName.substr(fileName.size() - 4) : std::string();
  for (char& ch : ext) ch = (char)std::tolower((unsigned char)ch);
  if (ext != ".stl") errorMessage("Reader: file format not supported");
  long long n = 0;
  check(aslb_read_stl(fileName.c_str(), nullptr, 0, &n), "readSurface");
  if (n < 1) errorMessage("readSurface: empty surface");
  std::vector<float> tri((size_t)n * 9);
  check(aslb_read_stl(fileName.c_str(), tri.data(), n, &n), "readSurface");
  for (size_t v = 0; v < tri.size(); v += 3) std::swap(tri[v], tri[v + 2]);
  return tri;
}
inline SPDataWithGhostNodesACLData sample_surface(const std::vector<float>& tri, const AVec<int>& size,
                                                  const AVec<>& pos0, double dx, double offset, double scale) {
  if (nD(size) != 3 || minComponent(size) < 3) errorMessage("readSurface: the sampled grid has no interior");
  std::vector<float> m((size_t)size[0] * size[1] * size[2]);
  const double p0[3] = {pos0[0], pos0[1], pos0[2]};
  check(aslb_surface_map(tri.data(), (long long)(tri.size() / 9), size[0], size[1], size[2], p0, dx, 4.0 * dx, 0,
                         offset, scale, m.data()),
        "readSurface");
  auto d = std::make_shared<DataWithGhostNodesACLData>(
      Block(size - AVec<int>(3, 2), dx, pos0 + AVec<>(3, dx)), 1u, 1u, acl::TYPE_FLOAT);
  std::vector<double>& v = d->values();
  for (size_t i = 0; i < m.size(); ++i) v[i] = m[i];
  return d;
}
inline SPDataWithGhostNodesACLData surface_on_bounds(const std::vector<float>& tri, double dx, const double* off) {
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) lo[a] = hi[a] = tri[a];
  for (size_t v = 0; v < tri.size(); v += 3)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], (double)tri[v + a]);
      hi[a] = std::max(hi[a], (double)tri[v + a]);
    }
  AVec<int> size(3);
  AVec<> pos0(3);
  for (int a = 0; a < 3; ++a) {
    const double ext = hi[a] - lo[a];
    const double l = off ? lo[a] - ext * off[2 * a] : lo[a] - 3.6 * dx;
    const double h = off ? hi[a] + ext * off[2 * a + 1] : hi[a] + 3.6 * dx;
    size[a] = int(std::floor((h - l) / dx)) + 1;
    pos0[a] = l;
  }
  return sample_surface(tri, size, pos0, dx, 1.8 * dx, 1.8 * dx);
}
}  // namespace aslb_detail

inline SPDataWithGhostNodesACLData readSurface(const std::string& fileName, Block& b) {
  return aslb_detail::sample_surface(aslb_detail::surface_triangles(fileName), b.getSize(), b.position, b.dx,
                                     1.2 * b.dx, 1.8 * b.dx);
}
inline SPDataWithGhostNodesACLData readSurface(const std::string& fileName, double dx) {
  return aslb_detail::surface_on_bounds(aslb_detail::surface_triangles(fileName), dx, nullptr);
}
inline SPDataWithGhostNodesACLData readSurface(const std::string& fileName, double dx, double offset_X0,
                                               double offset_XE, double offset_Y0, double offset_YE,
                                               double offset_Z0, double offset_ZE) {
  const double off[6] = {offset_X0, offset_XE, offset_Y0, offset_YE, offset_Z0, offset_ZE};
  return aslb_detail::surface_on_bounds(aslb_detail::surface_triangles(fileName), dx, off);
}

}  // namespace asl

#endif  // ASLB_ASL_IO_HPP
