// tri_host_input.cpp -- configuration, input files and preprocessing of the
// drop-in host.  Behaviour follows the reference's readers so the same .cfg
// and inputs give the same arrays (citations: reference project files).
#include <limits.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>

#include "tri_host.h"

namespace trihost {

std::string trim(std::string s) {
  auto notsp = [](unsigned char ch) { return !std::isspace(ch); };
  s.erase(std::find_if(s.rbegin(), s.rend(), notsp).base(), s.end());
  s.erase(s.begin(), std::find_if(s.begin(), s.end(), notsp));
  return s;
}

// std::getline splitting: a trailing delimiter does not yield an empty item
// (string_utils.h:200-216).
std::vector<std::string> split(const std::string& s, char delim) {
  std::vector<std::string> out;
  std::stringstream ss(s);
  std::string item;
  while (std::getline(ss, item, delim)) out.push_back(item);
  return out;
}

static std::string unquote(std::string v) {
  if (!v.empty() && v[0] == '"' && v[v.size() - 1] == '"' && v.size() >= 2) v = v.substr(1, v.size() - 2);
  return v;
}

// '#' comment handling of the reference: only the '#' character itself is
// removed, and not when it follows a quote (config_utils.h:211-216).
static void drop_hash(std::string& line) {
  size_t p = line.find('#');
  if (p != std::string::npos && p > 0 && line[p - 1] != '\'' && line[p - 1] != '"') line.erase(line.begin() + p);
}

std::map<std::string, std::string> parse_cfg(const std::string& content) {
  std::map<std::string, std::string> m;
  std::istringstream in(content);
  std::string line;
  while (std::getline(in, line)) {
    line = trim(line);
    if (line.empty() || line[0] == '#') continue;
    drop_hash(line);
    std::vector<std::string> kv = split(line, '=');
    if (kv.size() < 2) throw InputError("Error parsing configuration line: " + line);
    std::string key = kv[0], value = unquote(kv[1]);
    for (size_t i = 2; i < kv.size(); i++) value += kv[i];
    m.insert({key, value});  // the first occurrence of a key wins (std::map::insert)
  }
  return m;
}

static std::string argd(const std::map<std::string, std::string>& m, const std::string& k, const std::string& d = "") {
  auto it = m.find(k);
  return it == m.end() ? d : it->second;
}

template <typename T>
static std::vector<T> to_vec(const std::string& csv) {
  std::vector<T> out;
  for (const std::string& item : split(csv, ',')) {
    std::istringstream iss(item);
    T v{};
    iss >> v;
    out.push_back(v);
  }
  return out;
}

// Location files: "x,y" rows, '%' comment lines (config_utils.h:241-302).
static void read_locations(const std::string& path, std::vector<double>& xs, std::vector<double>& ys) {
  std::ifstream f(path);
  if (!f.good()) throw InputError("Error reading file: " + path);
  std::string line, sx, sy;
  while (std::getline(f, line)) {
    line = trim(line);
    if (line.empty() || line[0] == '%') continue;
    drop_hash(line);
    std::vector<std::string> kv = split(line, ',');
    if (kv.size() < 2) throw InputError("Error reading file: " + path + " (expected x,y)");
    sx += "," + unquote(kv[0]);
    sy += "," + unquote(kv[1]);
  }
  if (sx.empty()) return;
  xs = to_vec<double>(sx.substr(1));
  ys = to_vec<double>(sy.substr(1));
}

// External boundary file: type,x1,y1,x2,y2[,file or value] (config_utils.h:305-419).
static void read_extbc_file(const std::string& path, const std::string& dir, Args& a) {
  std::ifstream f(path);
  if (!f.good()) throw InputError("Error reading file: " + path);
  std::string line;
  while (std::getline(f, line)) {
    line = trim(line);
    if (line.empty() || line[0] == '%') continue;
    drop_hash(line);
    std::vector<std::string> kv = split(line, ',');
    if (kv.size() < 5) throw InputError("Error reading file: " + path + " (expected type,x1,y1,x2,y2[,bc])");
    int type = std::atoi(kv[0].c_str());
    std::string bc = type != 0 ? (kv.size() > 5 ? unquote(kv[5]) : std::string()) : std::string("0.0");
    a.ebc_type.push_back(to_vec<int>(unquote(kv[0]))[0]);
    a.ebc_x1.push_back(to_vec<double>(unquote(kv[1]))[0]);
    a.ebc_y1.push_back(to_vec<double>(unquote(kv[2]))[0]);
    a.ebc_x2.push_back(to_vec<double>(unquote(kv[3]))[0]);
    a.ebc_y2.push_back(to_vec<double>(unquote(kv[4]))[0]);
    a.ebc_fname.push_back(type == 1 ? dir + "/" + bc : bc);
  }
}

Args get_args(const std::string& cfg) {
  auto m = parse_cfg(cfg);
  Args a;
  a.outfile_pattern = argd(m, "outfile_pattern");
  a.hydrograph_filename = argd(m, "hydrograph_filename");
  a.runoff_filename = argd(m, "runoff_filename");
  a.dem_filename = argd(m, "dem_filename");
  a.src_loc_file = argd(m, "src_loc_file");
  a.runoff_map = argd(m, "runoff_map");
  a.observation_loc_file = argd(m, "observation_loc_file");
  a.extbc_file = argd(m, "extbc_file");
  a.extbc_dir = argd(m, "extbc_dir");
  a.const_mann = std::atof(argd(m, "const_mann").c_str());
  a.time_step = std::atof(argd(m, "time_step").c_str());
  a.time_increment_fixed = std::atoi(argd(m, "time_increment_fixed").c_str()) != 0;
  a.time_series_flag = std::atoi(argd(m, "time_series_flag").c_str()) != 0;
  a.courant = std::atof(argd(m, "courant").c_str());
  a.hextra = std::atof(argd(m, "hextra").c_str());
  a.gpu_direct_flag = std::atoi(argd(m, "gpu_direct_flag").c_str()) != 0;
  a.open_boundaries = std::atoi(argd(m, "open_boundaries").c_str()) != 0;
  a.num_sources = std::atoi(argd(m, "num_sources").c_str());
  a.num_runoffs = std::atoi(argd(m, "num_runoffs").c_str());
  a.num_extbc = std::atoi(argd(m, "num_extbc").c_str());
  a.checkpoint_id = std::atoi(argd(m, "checkpoint_id", "0").c_str());
  a.it_count = std::atoi(argd(m, "it_count", "0").c_str());
  a.it_print = std::atoi(argd(m, "it_print", "10000").c_str());
  std::string po = argd(m, "print_option");
  std::transform(po.begin(), po.end(), po.begin(), [](unsigned char c) { return (char)std::tolower(c); });
  a.print_option = po;
  a.max_value_print_option = argd(m, "max_value_print_option");
  a.input_format = argd(m, "input_format");
  a.input_option = argd(m, "input_option");
  a.output_format = argd(m, "output_format");
  a.output_option = argd(m, "output_option");
  a.projection = argd(m, "projection");
  a.h_infile = argd(m, "h_infile");
  a.qx_infile = argd(m, "qx_infile");
  a.qy_infile = argd(m, "qy_infile");
  a.n_infile = argd(m, "n_infile");
  a.domain_decomposition = argd(m, "domain_decomposition");
  a.factor_interval_domain_decomposition = std::atoi(argd(m, "factor_interval_domain_decomposition").c_str());
  a.sim_start_time = std::atof(argd(m, "sim_start_time").c_str());
  a.sim_duration = std::atof(argd(m, "sim_duration").c_str());
  std::string pi = argd(m, "print_interval");
  a.print_observation = std::atof(argd(m, "print_observation", pi).c_str());
  a.print_interval = std::atof(pi.c_str());
  a.input_folder = argd(m, "input_folder", "input");
  a.output_folder = argd(m, "output_folder", "output");
  if (a.num_sources > 0) read_locations(a.src_loc_file, a.src_x, a.src_y);
  if (a.time_series_flag) read_locations(a.observation_loc_file, a.obs_x, a.obs_y);
  if (a.num_extbc > 0) read_extbc_file(a.extbc_file, a.extbc_dir, a);
  if (a.input_option.empty()) a.input_option = "SEQ";
  if (a.input_option == "PAR") a.header_filename = argd(m, "header_filename");
  return a;
}

std::string read_file(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in.is_open()) throw InputError("Error reading file: " + path);
  std::stringstream ss;
  ss << in.rdbuf();
  return ss.str();
}

// The project directory is the executable's path two levels up
// (config_utils.h:542-580).
std::string root_dir(const char* p) {
  if (p == nullptr || *p == '\0') {
    char cwd[PATH_MAX];
    return getcwd(cwd, sizeof(cwd)) ? std::string(cwd) : std::string(".");
  }
  std::string path(p);
  if (path[0] != '/') {
    char cwd[PATH_MAX];
    if (getcwd(cwd, sizeof(cwd))) path = std::string(cwd) + "/" + path;
  }
  while (path.size() > 1 && path.back() == '/') path.pop_back();
  for (int i = 0; i < 2; i++) {
    size_t pos = path.find_last_of('/');
    if (pos == std::string::npos || pos == 0) break;
    path = path.substr(0, pos);
  }
  return path.empty() ? std::string(".") : path;
}

// ---- rasters --------------------------------------------------------------
DemHeader read_dem_header(const std::string& path, bool ascii) {
  DemHeader h;
  if (ascii) {  // dem_utils.h:163-228: last token of each of the first 6 lines
    std::ifstream f(path);
    if (!f.good()) throw InputError("Error reading file: " + path);
    std::string line;
    for (int ln = 1; ln <= 6 && std::getline(f, line); ln++) {
      line = trim(line);
      std::vector<std::string> t = split(line, ' ');
      if (t.empty() || line[0] == '#') continue;
      const char* v = t.back().c_str();
      switch (ln) {
        case 1: h.ncols = std::atoi(v); break;
        case 2: h.nrows = std::atoi(v); break;
        case 3: h.xll = std::atof(v); break;
        case 4: h.yll = std::atof(v); break;
        case 5: h.cell = std::atof(v); break;
        case 6: h.nodata = std::atoi(v); break;
      }
    }
  } else {  // dem_utils.h:231-290: 6 values of the raster type
    std::ifstream f(path, std::ios::binary);
    if (!f.good()) throw InputError("Error reading file: " + path);
    double v[6] = {0, 0, 0, 0, 0, 0};
    f.read(reinterpret_cast<char*>(v), sizeof(v));
    h.ncols = (int)v[0];
    h.nrows = (int)v[1];
    h.xll = v[2];
    h.yll = v[3];
    h.cell = v[4];
    h.nodata = (int)v[5];
  }
  return h;
}

// One text row: single-space separated; a token with '.' is read with atof,
// otherwise atoi (matrix_io.h:116-130).
template <typename T>
static void parse_row(const std::string& line, T* out, int cols, int row, const std::string& path) {
  std::vector<std::string> tok = split(line, ' ');
  int j = 0;
  for (const std::string& v : tok) {
    if (j > cols - 1)
      throw InputError("Error reading file: " + path + ". More than one space as separator?. Check row " +
                       std::to_string(row + 1));
    out[j++] = v.find('.') != std::string::npos ? (T)std::atof(v.c_str()) : (T)std::atoi(v.c_str());
  }
}

template <typename T>
static std::vector<T> read_ascii(const std::string& path, int rows, int cols, int header_lines, bool check_dims) {
  std::ifstream f(path);
  if (!f.is_open()) throw InputError("Error reading file: " + path);
  std::vector<std::string> lines;
  std::string line;
  while (std::getline(f, line)) lines.push_back(line);
  if (check_dims) {  // get_dims_2d: columns of the first line, number of lines (matrix.h:1011-1040)
    int ncol = lines.empty() ? 0 : (int)split(lines[0], ' ').size();
    int nrow = (int)lines.size();
    if (nrow != rows || ncol != cols)
      throw InputError("Invalid dimension of " + path + ". (row,col): (" + std::to_string(nrow) + "," +
                       std::to_string(ncol) + ")");
  }
  std::vector<T> out((size_t)rows * cols, T(0));
  int i = 0;
  for (size_t k = header_lines; k < lines.size() && i < rows; k++, i++)
    parse_row<T>(lines[k], out.data() + (size_t)i * cols, cols, i, path);
  return out;
}

template <typename T>
static std::vector<T> read_binary(const std::string& path, int rows, int cols, int header_values, bool check) {
  std::ifstream f(path, std::ios::binary);
  if (!f.is_open()) throw InputError("Error reading file: " + path);
  std::vector<T> hdr(header_values);
  f.read(reinterpret_cast<char*>(hdr.data()), sizeof(T) * header_values);
  if (check && ((int)hdr[0] != rows || (int)hdr[1] != cols)) throw InputError("Invalid Matrix dimensions");
  std::vector<T> out((size_t)rows * cols);
  f.read(reinterpret_cast<char*>(out.data()), sizeof(T) * out.size());
  if ((size_t)f.gcount() != sizeof(T) * out.size()) throw InputError("Error reading file: " + path + " (short file)");
  return out;
}

std::vector<double> read_dem(const std::string& path, int rows, int cols, bool ascii) {
  return ascii ? read_ascii<double>(path, rows, cols, 6, false) : read_binary<double>(path, rows, cols, 6, false);
}
std::vector<double> read_raster(const std::string& path, int rows, int cols, bool ascii) {
  return ascii ? read_ascii<double>(path, rows, cols, 0, true) : read_binary<double>(path, rows, cols, 2, true);
}
std::vector<int32_t> read_raster_int(const std::string& path, int rows, int cols, bool ascii) {
  return ascii ? read_ascii<int32_t>(path, rows, cols, 0, true) : read_binary<int32_t>(path, rows, cols, 2, true);
}

std::vector<std::vector<double>> read_table(const std::string& path) {
  std::ifstream f(path);
  if (!f.good()) throw InputError("Error reading file: " + path);
  std::vector<std::vector<double>> rows;
  std::string line;
  while (std::getline(f, line)) {
    line = trim(line);
    std::vector<std::string> parts = split(line, '%');
    std::string body = parts.empty() ? std::string() : trim(parts[0]);
    if (!body.empty()) rows.push_back(to_vec<double>(body));
  }
  return rows;
}

// ---- preprocessing ---------------------------------------------------------
static std::vector<double> pad(const std::vector<double>& a, int r, int c, double ghost) {
  std::vector<double> o((size_t)(r + 2) * (c + 2), ghost);
  for (int i = 0; i < r; i++)
    std::copy(a.begin() + (size_t)i * c, a.begin() + (size_t)(i + 1) * c, o.begin() + (size_t)(i + 1) * (c + 2) + 1);
  return o;
}

// matrix<T>::copy_value_into_ghost_cells (matrix.h:848-865)
static void copy_ghosts(std::vector<double>& a, int R, int C) {
  for (int i = 0; i < R; i++) {
    a[(size_t)i * C] = a[(size_t)i * C + 1];
    a[(size_t)i * C + C - 1] = a[(size_t)i * C + C - 2];
  }
  for (int j = 0; j < C; j++) {
    a[j] = a[(size_t)C + j];
    a[(size_t)(R - 1) * C + j] = a[(size_t)(R - 2) * C + j];
  }
}

static int src_col(double x, double xll, double cell) { return (int)std::ceil(((x - xll) / cell) + 1e-16) - 1; }
static int src_row(double y, double yll, double cell, int nrows) {
  return (int)std::ceil((nrows - ((y - yll) / cell)) + 1e-16) - 1;
}

static std::string two(int v) { return v < 10 ? "0" + std::to_string(v) : std::to_string(v); }

// Partitioned input (input_option=PAR, triton_init.h:359-717): raster <base>
// is stored as <base>_NN<ext>, one file per partition (NN: the rank, two
// digits), without the DEM header (that comes from header_filename).  A
// single rank reads _00 holding the whole domain.  Files written for N ranks
// hold row slabs as create_local_dims makes them (mpi_utils.h:73-89: R/N
// rows each, one more for each of the first R%N ranks); they are read in rank
// order and stacked, so a case partitioned for N ranks runs on one GPU.
template <typename T, typename Reader>
static std::vector<T> read_parts(const std::string& base, const std::string& ext, int R, int C, Reader read) {
  int n = 0;
  while (n < 100 && std::ifstream(base + "_" + two(n) + ext).good()) n++;
  if (n == 0) throw InputError("Error reading file: " + base + "_00" + ext);
  std::vector<T> out;
  out.reserve((size_t)R * C);
  for (int p = 0; p < n; p++) {
    const int rows = R / n + (p < R % n ? 1 : 0);
    const std::vector<T> part = read(base + "_" + two(p) + ext, rows, C);
    out.insert(out.end(), part.begin(), part.end());
  }
  return out;
}

Problem load_problem(const std::string& argv0, const std::string& cfg_arg, int checkpoint_id) {
  Problem P;
  P.project_dir = root_dir(argv0.c_str());
  // read_configuration (triton_init.h:85-136): a numeric first argument is
  // not a cfg path; a checkpoint id selects the checkpoint's cfg
  std::string cfg_path = P.project_dir + "/input/cfg/case4.cfg";
  bool numeric = false;
  {
    std::stringstream conv(cfg_arg);
    double tmp;
    conv >> tmp;
    numeric = !cfg_arg.empty() && conv.eof() && !conv.fail();
  }
  if (!cfg_arg.empty() && !numeric) cfg_path = cfg_arg;
  // The reference composes this path from the output folder before any cfg
  // has been read, i.e. from an empty folder name (triton_init.h:98-101):
  // <project>//cfg/config_<id>.cfg, not <project>/<output_folder>/cfg where
  // the run wrote it; the rasters it then names come from <output_folder>.
  if (checkpoint_id > 0)
    cfg_path = P.project_dir + "//cfg/config_" + std::to_string(checkpoint_id) + ".cfg";
  P.cfg_content = read_file(cfg_path);
  Args& a = P.args;
  a = get_args(P.cfg_content);
  P.simtime = a.sim_start_time;
  const bool par = a.input_option == "PAR";
  if (!par && a.input_option != "SEQ")
    throw InputError("input_option=" + a.input_option + " is not supported (SEQ or PAR)");
  const bool asc = a.input_format == "ASC";
  auto raster_part = [asc](const std::string& path, int r, int c) { return read_raster(path, r, c, asc); };

  // read_inflows (triton_init.h:140-167)
  std::vector<std::vector<double>> hyg, roff;
  if (a.num_sources > 0) {
    hyg = read_table(a.hydrograph_filename);
    for (auto& r : hyg) r[0] = r[0] * 3600.0;
  }
  if (a.num_runoffs > 0) {
    roff = read_table(a.runoff_filename);
    const int nin = roff.empty() ? 0 : (int)roff.back().size() - 1;
    for (auto& r : roff) r[0] = r[0] * 3600.0;
    for (int i = 0; i < nin; i++)
      for (auto& r : roff) r[i + 1] /= 3600.0;
    for (int i = 0; i < nin; i++)
      for (auto& r : roff) r[i + 1] *= 0.001;
  }

  // DEM and fields (triton_init.h:171-353)
  // the header of a partitioned DEM is its own ASCII file (triton_init.h:171-191)
  P.dem = par ? read_dem_header(a.header_filename, true) : read_dem_header(a.dem_filename, asc);
  const int R = P.dem.nrows, C = P.dem.ncols;
  if (R <= 0 || C <= 0) throw InputError("Invalid DEM dimensions in " + (par ? a.header_filename : a.dem_filename));
  const int Rp = R + 2, Cp = C + 2;
  P.rows = Rp;
  P.cols = Cp;
  if (par)  // DEM partitions: ASCII without a header and unchecked, binary with its two-value header
    P.z = pad(read_parts<double>(a.dem_filename, ".dem", R, C,
                                 [asc](const std::string& path, int r, int c) {
                                   return asc ? read_ascii<double>(path, r, c, 0, false)
                                              : read_binary<double>(path, r, c, 2, true);
                                 }),
              R, C, 0.0);
  else
    P.z = pad(read_dem(a.dem_filename, R, C, asc), R, C, 0.0);
  if (!a.open_boundaries) {  // closed walls: DEM ghosts 1e6 (matrix.h:929-945)
    for (int i = 0; i < Rp; i++) P.z[(size_t)i * Cp] = P.z[(size_t)i * Cp + Cp - 1] = 1e6;
    for (int j = 0; j < Cp; j++) P.z[j] = P.z[(size_t)(Rp - 1) * Cp + j] = 1e6;
  } else {
    copy_ghosts(P.z, Rp, Cp);
  }
  std::vector<double> nin;
  if (!a.n_infile.empty()) {
    nin = par ? read_parts<double>(a.n_infile, ".mann", R, C, raster_part) : read_raster(a.n_infile, R, C, asc);
  } else {
    nin.assign((size_t)R * C, 0.0);
    for (double& v : nin) v = v + a.const_mann;
  }
  P.n2 = pad(nin, R, C, 0.0);
  copy_ghosts(P.n2, Rp, Cp);
  for (double& v : P.n2) v = v * v;
  auto field = [&](const std::string& f) {
    if (f.empty()) return std::vector<double>((size_t)Rp * Cp, 0.0);
    std::vector<double> v =
        pad(par ? read_parts<double>(f, ".out", R, C, raster_part) : read_raster(f, R, C, asc), R, C, 0.0);
    if (a.open_boundaries) copy_ghosts(v, Rp, Cp);
    return v;
  };
  P.h = field(a.h_infile);
  P.qx = field(a.qx_infile);
  P.qy = field(a.qy_infile);
  std::vector<int32_t> rin;
  if (!a.runoff_map.empty()) {
    std::vector<int32_t> r =
        par ? read_parts<int32_t>(a.runoff_map, ".rmap", R, C,
                                  [asc](const std::string& path, int rr, int cc) {
                                    return read_raster_int(path, rr, cc, asc);
                                  })
            : read_raster_int(a.runoff_map, R, C, asc);
    rin.assign((size_t)Rp * Cp, 0);
    for (int i = 0; i < R; i++)
      for (int j = 0; j < C; j++) rin[(size_t)(i + 1) * Cp + j + 1] = r[(size_t)i * C + j];
  }
  bool have_maxh = false;
  // Checkpoint rasters.  Sequential input reads <what>_<id>_00.out holding the
  // whole domain, and only when output_option is SEQ (triton_init.h:303-353;
  // otherwise the initial fields stand).  Partitioned input reads one file per
  // rank, <what>_<id>_<rank>.out with that rank's rows (triton_init.h:577-626):
  // files written by N ranks are stacked in rank order like the other
  // partitioned rasters.
  if (a.checkpoint_id > 0 && (par || a.output_option == "SEQ")) {
    const std::string t = two(a.checkpoint_id);
    const std::string base = P.project_dir + "/" + a.output_folder + "/bin/";
    auto hot = [&](const std::string& what) {
      std::vector<double> v =
          pad(par ? read_parts<double>(base + what + "_" + t, ".out", R, C,
                                       [](const std::string& path, int r, int c) {
                                         return read_raster(path, r, c, false);
                                       })
                  : read_raster(base + what + "_" + t + "_00.out", R, C, false),
              R, C, 0.0);
      if (a.open_boundaries) copy_ghosts(v, Rp, Cp);
      return v;
    };
    P.h = hot("H");
    P.qx = hot("QX");
    P.qy = hot("QY");
    if (!a.max_value_print_option.empty()) {
      P.maxh = hot("MH");
      have_maxh = true;
    }
  }
  if (!have_maxh) P.maxh = P.h;

  // sources (triton_init.h:723-816)
  if (a.num_sources > 0) {
    if ((int)a.src_x.size() < a.num_sources || (int)a.src_y.size() < a.num_sources)
      throw InputError("Fewer source locations than num_sources");
    for (int i = 0; i < a.num_sources; i++) {
      int c = src_col(a.src_x[i], P.dem.xll, P.dem.cell);
      int r = src_row(a.src_y[i], P.dem.yll, P.dem.cell, R);
      if (c >= C || r >= R || c < 0 || r < 0) throw InputError("Source " + std::to_string(i + 1) + " is out of bounds");
      P.src_cells.push_back((r + 1) * Cp + c + 1);
    }
    if (hyg.size() < 2) throw InputError("Inflow or runoff index out of bounds: 1 out of " + std::to_string(hyg.size()));
    P.nsrc = a.num_sources;
    P.hyg_rows = (int)hyg.size();
    for (auto& row : hyg) {
      if ((int)row.size() < P.nsrc + 1) throw InputError("Hydrograph row has fewer columns than sources");
      P.hyg_t.push_back(row[0]);
    }
    for (auto& row : hyg)
      for (int j = 0; j < P.nsrc; j++) P.hyg_v.push_back(row[j + 1]);
  }
  // observations (triton_init.h:818-911)
  if (a.time_series_flag) {
    for (size_t i = 0; i < a.obs_x.size(); i++) {
      int c = src_col(a.obs_x[i], P.dem.xll, P.dem.cell);
      int r = src_row(a.obs_y[i], P.dem.yll, P.dem.cell, R);
      if (c >= C || r >= R || c < 0 || r < 0)
        throw InputError("Observation " + std::to_string(i + 1) + " is out of bounds");
      P.obs_cells.push_back((r + 1) * Cp + c + 1);
    }
  }
  // external boundaries (triton_init.h:913-1055, extbc.h:206-294)
  if (a.num_extbc > 0) {
    int start = 0;
    for (int i = 0; i < a.num_extbc; i++) {
      if (i >= (int)a.ebc_type.size()) throw InputError("Fewer external boundaries than num_extbc");
      const int bt = a.ebc_type[i];
      std::vector<std::vector<double>> data;
      if (bt == 1) {
        data = read_table(a.ebc_fname[i]);
        for (auto& r : data) r[0] = r[0] * 3600.0;
      } else {
        std::istringstream iss(a.ebc_fname[i]);
        double v = 0;
        iss >> v;
        data.push_back({v, v});
      }
      if (data.empty()) throw InputError("Empty external boundary table " + a.ebc_fname[i]);
      int c1 = src_col(a.ebc_x1[i], P.dem.xll, P.dem.cell), r1 = src_row(a.ebc_y1[i], P.dem.yll, P.dem.cell, R);
      int c2 = src_col(a.ebc_x2[i], P.dem.xll, P.dem.cell), r2 = src_row(a.ebc_y2[i], P.dem.yll, P.dem.cell, R);
      if (c1 >= C || c2 >= C)
        throw InputError("Please revise x-coordinates of the external BC. It must be at the boundary of the domain");
      if (r1 >= R || r2 >= R)
        throw InputError("Please revise y-coordinates of the external BC. It must be at the boundary of the domain");
      auto on_edge = [&](int c, int r) { return c == 0 || c == C - 1 || r == 0 || r == R - 1; };
      if (!on_edge(c1, r1) || !on_edge(c2, r2))
        throw InputError("Error selecting the external BC. It must be at the boundary of the domain");
      if (c1 != c2 && r1 != r2)
        throw InputError("Error selecting the external BC. The points must be aligned with a boundary of the domain");
      const int n = c1 == c2 ? std::abs(r1 - r2) + 1 : std::abs(c1 - c2) + 1;
      const int cmin = std::min(c1, c2), cmax = std::max(c1, c2), rmin = std::min(r1, r2), rmax = std::max(r1, r2);
      int loc = -1;
      if (cmin == cmax) loc = cmin == 0 ? 0 : 2;
      if (rmin == rmax) loc = rmin == 0 ? 1 : 3;
      for (int k = 0; k < n; k++) {
        int ic = 0, ir = 0;
        if (loc == 0) { ic = 0; ir = rmin + k; }
        if (loc == 2) { ic = C - 1; ir = rmin + k; }
        if (loc == 1) { ic = cmin + k; ir = 0; }
        if (loc == 3) { ic = cmin + k; ir = R - 1; }
        // DEM ghost next to the boundary cell (matrix.h:869-926)
        const int ix = ir + 1, iy = ic + 1;
        const double v = P.z[(size_t)ix * Cp + iy];
        if (loc == 0) P.z[(size_t)ix * Cp + iy - 1] = v;
        if (loc == 2) P.z[(size_t)ix * Cp + iy + 1] = v;
        if (loc == 1) P.z[(size_t)(ix - 1) * Cp + iy] = v;
        if (loc == 3) P.z[(size_t)(ix + 1) * Cp + iy] = v;
        if (ir == 0 && ic == 0) P.z[0] = P.z[1] = P.z[(size_t)Cp] = v;
        if (ir == 0 && ic == Cp - 3) P.z[(size_t)Cp - 2] = P.z[(size_t)Cp - 1] = P.z[(size_t)2 * Cp - 1] = v;
        if (ir == Rp - 3 && ic == 0)
          P.z[(size_t)(Rp - 2) * Cp] = P.z[(size_t)(Rp - 1) * Cp] = P.z[(size_t)(Rp - 1) * Cp + 1] = v;
        if (ir == Rp - 3 && ic == Cp - 3)
          P.z[(size_t)(Rp - 2) * Cp + Cp - 1] = P.z[(size_t)(Rp - 1) * Cp + Cp - 2] =
              P.z[(size_t)(Rp - 1) * Cp + Cp - 1] = v;
        P.bc_cells.push_back(ix * Cp + iy);
        P.bc_types.push_back(bt);
        P.bc_start.push_back(start);
        P.bc_nrows.push_back((int)data.size());
      }
      for (auto& r : data) {
        if (r.size() < 2) throw InputError("External boundary table row needs two values: " + a.ebc_fname[i]);
        P.bc_v1.push_back(r[0]);
        P.bc_v2.push_back(r[1]);
      }
      start += (int)data.size();
    }
    // ghost copies of DEM/h/qx/qy next to boundary cells (triton_init.h:1250-1289)
    for (int32_t ii : P.bc_cells) {
      const int ix = ii / Cp, iy = ii % Cp;
      std::vector<int> nb;
      if (iy == 1) nb.push_back(ii - 1);
      if (iy == Cp - 2) nb.push_back(ii + 1);
      if (ix == 1) nb.push_back(ii - Cp);
      if (ix == Rp - 2) nb.push_back(ii + Cp);
      for (int g : nb) {
        P.z[g] = P.z[ii];
        P.h[g] = P.h[ii];
        P.qx[g] = P.qx[ii];
        P.qy[g] = P.qy[ii];
      }
    }
  }
  // runoff (triton_init.h:1299-1357)
  if (a.num_runoffs > 0) {
    if (roff.size() < 2) throw InputError("Inflow or runoff index out of bounds: 1 out of " + std::to_string(roff.size()));
    P.nroff = a.num_runoffs;
    P.roff_rows = (int)roff.size();
    for (int j = 0; j + 1 < P.roff_rows; j++)
      if (P.simtime > roff[j][0] && P.simtime <= roff[j + 1][0]) P.runoff_row = j;
    for (auto& r : roff) P.roff_t.push_back(r[0]);
    P.roff_v.assign((size_t)P.nroff * P.roff_rows, 0.0);
    for (int j = 0; j < P.nroff; j++)
      for (int k = 0; k < P.roff_rows; k++) {
        if ((int)roff[k].size() < j + 2) throw InputError("Runoff row has fewer columns than num_runoffs");
        P.roff_v[(size_t)j * P.roff_rows + k] = roff[k][j + 1];
      }
    if (rin.empty()) rin.assign((size_t)Rp * Cp, 0);
    P.zone = rin;
  }
  // compute_init_dt (triton_simulate.h:163-187)
  double idt = a.time_series_flag ? std::fmin(a.print_observation, a.print_interval) : a.print_interval;
  if (a.num_runoffs > 0) idt = std::fmin(idt, P.roff_t[1] - P.roff_t[0]);
  if (P.nsrc > 0) idt = std::fmin(idt, P.hyg_t[1] - P.hyg_t[0]);
  P.init_dt = idt * 0.01;
  return P;
}

}  // namespace trihost
