// tri_host_main.cpp -- the drop-in executable: `triton_b200 <cfg> [nthreads]
// [checkpoint_id]`, the command line of the reference's triton.exe
// (triton_init.h:17-27).  It reads the same configuration and inputs, runs the
// time loop on the GPU through the C ABI, and writes the same files
// (binary/ASCII rasters, observation series, restart cfg, cid, performance
// summaries) as triton<T>::simulate (triton_simulate.h:12-160).
#include <dirent.h>
#include <sys/stat.h>
#include <sys/time.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <future>
#include <iomanip>
#include <iostream>
#include <limits>
#include <sstream>
#include <thread>

#include "tri_fixed6.h"
#include "tri_host.h"
#include "triton_b200.h"

using namespace trihost;

namespace {

#define C_RESET "\033[0m"
#define C_RED "\033[31m"
#define C_GREEN "\033[32m"
#define C_BLUE "\033[34m"
#define C_GRAY "\033[90m"

struct ApiError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void ok(int rc, const char* what) {
  if (rc != TRI_OK) throw ApiError(std::string(what) + ": " + tri_last_error());
}

void ensure_dir(const std::string& d) {
  DIR* p = opendir(d.c_str());
  if (p) {
    closedir(p);
    return;
  }
  mkdir(d.c_str(), S_IRWXU);
}

// Wall-clock timers with the reference's categories (supertimer.h, constants.h:127-133).
struct Timers {
  using clk = std::chrono::steady_clock;
  std::map<std::string, double> total;
  std::map<std::string, clk::time_point> t0;
  void start(const std::string& k) { t0[k] = clk::now(); }
  void stop(const std::string& k) {
    auto it = t0.find(k);
    if (it == t0.end()) return;
    total[k] += std::chrono::duration<double>(clk::now() - it->second).count();
    t0.erase(it);
  }
  double get(const std::string& k) { return total.count(k) ? total[k] : 0.0; }
};

struct Output {
  const Problem& P;
  std::string root;  // project_dir/output_folder
  int threads = 1;   // host threads formatting ASCII rasters
  explicit Output(const Problem& p) : P(p), root(p.project_dir + "/" + p.args.output_folder) {}

  std::string mat_path(const std::string& what, const std::string& sub, int print_id) const {
    std::string fmt = P.args.outfile_pattern + ".out";
    char buf[256];
    std::snprintf(buf, sizeof(buf), fmt.c_str(), root.c_str(), sub.c_str(), what.c_str(), print_id, 0);
    return std::string(buf);
  }
  // write_output_binary_sequential (output_binary.h:12-87): rows, cols as T, interior rows
  void binary(const std::vector<double>& a, const std::string& what, int print_id) const {
    ensure_dir(root + "/");
    ensure_dir(root + "/bin/");
    std::ofstream f(mat_path(what, "bin", print_id), std::ios::binary);
    const int R = P.rows, C = P.cols;
    double hr = R - 2, hc = C - 2;
    f.write(reinterpret_cast<const char*>(&hr), sizeof(double));
    f.write(reinterpret_cast<const char*>(&hc), sizeof(double));
    for (int i = 1; i < R - 1; i++) f.write(reinterpret_cast<const char*>(&a[(size_t)i * C + 1]), (C - 2) * sizeof(double));
  }
  // write_output_ascii_sequential (output_ascii.h:12-81): fixed, 6 decimals,
  // one line per interior row.  Bands of rows are formatted on 'threads'
  // threads (trihost::append_fixed6 gives printf's "%.6f" text) and written
  // in row order.
  void ascii(const std::vector<double>& a, const std::string& what, int print_id) const {
    ensure_dir(root + "/");
    ensure_dir(root + "/asc/");
    FILE* f = std::fopen(mat_path(what, "asc", print_id).c_str(), "w");
    if (!f) return;
    const int R = P.rows, C = P.cols, nt = std::max(1, threads);
    const int band = std::max(1, std::min(256, (R - 2 + nt - 1) / nt));
    auto format_rows = [&](int i0, int i1, std::string& text) {
      text.clear();
      text.reserve((size_t)(i1 - i0) * (size_t)(C - 2) * 10);
      for (int i = i0; i < i1; i++) {
        for (int j = 1; j < C - 1; j++) {
          trihost::append_fixed6(text, a[(size_t)i * C + j]);
          if (j < C - 2) text.push_back(' ');
        }
        text.push_back('\n');
      }
    };
    std::vector<std::string> parts((size_t)nt);
    for (int r0 = 1; r0 < R - 1; r0 += nt * band) {
      std::vector<std::thread> pool;
      for (int t = 0; t < nt; t++) {
        const int i0 = std::min(R - 1, r0 + t * band), i1 = std::min(R - 1, i0 + band);
        if (t == nt - 1)
          format_rows(i0, i1, parts[(size_t)t]);
        else
          pool.emplace_back(format_rows, i0, i1, std::ref(parts[(size_t)t]));
      }
      for (std::thread& th : pool) th.join();
      for (const std::string& text : parts) std::fwrite(text.data(), 1, text.size(), f);
    }
    std::fclose(f);
  }
  void write(const std::string& what, const std::vector<double>& a, int print_id) const {
    const std::string& fmt = P.args.output_format;
    if (fmt == "ASC") {
      binary(a, what, print_id);
      ascii(a, what, print_id);
    } else if (fmt == "BIN") {
      binary(a, what, print_id);
    }  // GTIFF needs GDAL: this executable, like a reference build without TRITON_GDAL, does not write it
  }
  // output_cfg (output.h:754-811): the restart cfg with four keys rewritten
  void restart_cfg(double simtime, int print_id, double average_dt, int it_count) const {
    std::string s = P.cfg_content;
    std::istringstream ss(s);
    std::string line;
    auto fixed = [](double v) {
      std::ostringstream o;
      o << std::fixed << std::setprecision(std::numeric_limits<double>::max_digits10) << v;
      return o.str();
    };
    while (std::getline(ss, line)) {
      const char* keys[] = {"sim_start_time=", "checkpoint_id=", "time_step=", "it_count="};
      for (int k = 0; k < 4; k++) {
        if (line.find(keys[k]) == std::string::npos) continue;
        size_t pos = s.find(keys[k]);
        std::string v = k == 0 ? fixed(simtime) : k == 1 ? std::to_string(print_id) : k == 2 ? fixed(average_dt)
                                                                                        : std::to_string(it_count);
        s.replace(pos, line.length(), std::string(keys[k]) + v);
        break;
      }
    }
    ensure_dir(root + "/cfg/");
    std::ofstream f(root + "/cfg/config_" + std::to_string(print_id) + ".cfg");
    f << s;
  }
  // init_time_series headers (output.h:443-501)
  void series_headers(size_t nobs) const {
    ensure_dir(root + "/");
    ensure_dir(root + "/series/");
    if (P.args.checkpoint_id != 0) return;
    const char* keys[] = {"h", "u", "v"};
    const char* names[] = {"H", "QX", "QY"};
    for (int k = 0; k < 3; k++) {
      if (P.args.print_option.find(keys[k]) == std::string::npos) continue;
      std::string s = "Time(s)";
      for (size_t i = 0; i < nobs; i++) s += std::string(",") + names[k] + "_at_Point_" + std::to_string(i + 1);
      std::ofstream f(root + "/series/" + names[k] + "_at_Xsec.txt");
      f << s << "\n";
    }
  }
  // output_time_series (output_timeseries.h:12-47): std::to_string values
  void series(const std::vector<double>& h, const std::vector<double>& qx, const std::vector<double>& qy,
              double simtime) const {
    const char* keys[] = {"h", "u", "v"};
    const char* names[] = {"H", "QX", "QY"};
    const std::vector<double>* vals[] = {&h, &qx, &qy};
    for (int k = 0; k < 3; k++) {
      if (P.args.print_option.find(keys[k]) == std::string::npos) continue;
      std::string s = std::to_string(simtime);
      for (double v : *vals[k]) s += "," + std::to_string(v);
      std::ofstream f(root + "/series/" + names[k] + "_at_Xsec.txt", std::ios::app);
      f << s << "\n";
    }
    std::cerr << C_BLUE "[OBS]" C_RESET " Observation data written at time " << simtime << " seconds.\n";
  }
  // write_times (output.h:814-894)
  void times(Timers& t, int print_id) const {
    std::string path;
    if (print_id != -1) {
      ensure_dir(root + "/performance/");
      path = root + "/performance/performance" + std::to_string(print_id) + ".txt";
    } else {
      path = root + "/performance.txt";
    }
    const double comp = t.get("compute"), io = t.get("io"), sim = t.get("simulation"), tot = t.get("total");
    const double other = sim - comp - io, init = tot - sim;
    std::ofstream f(path);
    f << "%Rank, Compute, MPI, IO, Resize, Other, Simulation, Init, Total" << std::endl;
    f << std::setprecision(4) << 0 << ", " << comp << ", " << 0.0 << ", " << io << ", " << 0.0 << ", " << other
      << ", " << sim << ", " << init << ", " << tot << std::endl;
    f << std::setprecision(4) << "Average" << ", " << comp << ", " << 0.0 << ", " << io << ", " << 0.0 << ", "
      << other << ", " << sim << ", " << init << ", " << tot << std::endl;
  }
};

int run(int argc, char** argv) {
  Timers T;
  T.start("total");
  const std::string cfg_arg = argc > 1 ? argv[1] : "";
  const int ckpt = argc > 3 ? std::atoi(argv[3]) : 0;
  std::cerr << C_GRAY "[..] " C_RESET "Reading configuration file" << std::endl;
  Problem P = load_problem(argv[0], cfg_arg, ckpt);
  const Args& a = P.args;
  std::cerr << C_GREEN "[OK] " C_RESET "Configuration file read" << std::endl;

  tri_grid_desc g{};
  g.rows = P.rows;
  g.cols = P.cols;
  g.cell_size = P.dem.cell;
  g.courant = a.courant;
  g.hextra = a.hextra;
  g.open_boundaries = a.open_boundaries;
  const char* prec = std::getenv("TRITON_B200_PRECISION");
  g.precision = (prec && std::strcmp(prec, "fp32") == 0) ? TRI_FP32 : TRI_FP64;
  tri_domain* d = nullptr;
  ok(tri_domain_create(&g, nullptr, &d), "tri_domain_create");
  struct Guard {
    tri_domain* d;
    ~Guard() { tri_domain_destroy(d); }
  } guard{d};
  const int64_t n = (int64_t)P.rows * P.cols;
  ok(tri_domain_upload(d, TRI_FIELD_DEM, P.z.data(), n), "upload dem");
  ok(tri_domain_upload(d, TRI_FIELD_NMAN2, P.n2.data(), n), "upload manning");
  ok(tri_domain_upload(d, TRI_FIELD_H, P.h.data(), n), "upload h");
  ok(tri_domain_upload(d, TRI_FIELD_QX, P.qx.data(), n), "upload qx");
  ok(tri_domain_upload(d, TRI_FIELD_QY, P.qy.data(), n), "upload qy");
  ok(tri_domain_upload(d, TRI_FIELD_MAXH, P.maxh.data(), n), "upload maxh");
  if (P.nroff > 0)
    ok(tri_domain_set_runoff(d, P.nroff, P.roff_rows, P.roff_t.data(), P.roff_v.data(), P.zone.data(), n),
       "set runoff");
  if (P.nsrc > 0)
    ok(tri_domain_set_sources(d, P.nsrc, P.src_cells.data(), P.hyg_rows, P.hyg_t.data(), P.hyg_v.data()),
       "set sources");
  if (!P.bc_cells.empty())
    ok(tri_domain_set_extbc(d, (int32_t)P.bc_cells.size(), P.bc_cells.data(), P.bc_types.data(), P.bc_start.data(),
                            P.bc_nrows.data(), (int32_t)P.bc_v1.size(), P.bc_v1.data(), P.bc_v2.data()),
       "set extbc");
  if (!P.obs_cells.empty())
    ok(tri_domain_set_observations(d, (int32_t)P.obs_cells.size(), P.obs_cells.data()), "set observations");

  // simulate (triton_simulate.h:12-160)
  std::cerr << C_GREEN "[OK] " C_RESET "Simulation starts" << std::endl;
  T.start("simulation");
  Output out(P);
  // [nthreads] (the reference's OpenMP thread count) formats the ASCII rasters
  out.threads = argc > 2 ? std::max(1, std::atoi(argv[2]))
                         : (int)std::max(1u, std::thread::hardware_concurrency());
  double simtime = P.simtime;
  const size_t nobs = P.obs_cells.size();
  std::vector<double> oh(nobs), oqx(nobs), oqy(nobs);
  auto observe = [&]() {
    T.start("compute");
    if (nobs) ok(tri_domain_observe(d, oh.data(), oqx.data(), oqy.data()), "observe");
    T.stop("compute");
    T.start("io");
    out.series(oh, oqx, oqy, simtime);
    T.stop("io");
  };
  if (a.time_series_flag) {
    out.series_headers(a.obs_x.size());
    observe();
  }
  tri_clock c{};
  c.simtime = simtime;
  c.sim_duration = a.sim_duration;
  c.print_interval = a.print_interval;
  c.print_observation = a.print_observation;
  c.last_obs_time = simtime;
  c.init_dt = P.init_dt;
  c.time_step = a.time_step;
  c.average_dt = 0.0;
  c.global_dt = a.time_step;
  c.print_id = a.checkpoint_id;
  if (c.print_id == 0 && simtime > 0.0) c.print_id = (int)(simtime / a.print_interval);
  c.it_count = a.it_count;
  c.it_print = a.it_print;
  c.time_series = a.time_series_flag;
  c.time_increment_fixed = a.time_increment_fixed;
  c.runoff_row = P.runoff_row;
  c.src_idx_low = 0;
  ok(tri_domain_set_clock(d, &c), "set clock");
  int it_count_average = 0;
  std::vector<double> bh(n), bqx(n), bqy(n), bmh(n);
  // The rasters of an output time, its restart cfg and cid are written by a
  // background task while the GPU goes on stepping; the next output time
  // waits for it before it downloads into the same buffers (the cfg and cid
  // name a checkpoint only once its rasters are complete).
  std::future<void> writing;
  auto finish_writing = [&]() {
    if (!writing.valid()) return;
    T.start("io");
    writing.get();
    T.stop("io");
  };
  while (true) {
    T.start("compute");
    tri_progress p{};
    ok(tri_domain_advance(d, 1 << 30, &p), "advance");
    T.stop("compute");
    ok(tri_domain_get_clock(d, &c), "get clock");
    simtime = c.simtime;
    it_count_average += p.steps;
    if (p.events & TRI_EV_LOG) {
      std::cerr << C_GRAY "[INFO] " C_RESET " Time: " << simtime << "\tdt: " << c.average_dt / it_count_average
                << "\tit: " << c.it_count << std::endl;
      it_count_average = 0;
      c.average_dt = 0.0;
    }
    if (p.events & TRI_EV_OBS) {
      c.last_obs_time += c.print_observation;
      observe();
    }
    if (p.events & TRI_EV_PRINT) {
      c.print_id++;
      finish_writing();
      T.start("compute");
      ok(tri_domain_download(d, TRI_FIELD_H, bh.data(), n), "download h");
      ok(tri_domain_download(d, TRI_FIELD_QX, bqx.data(), n), "download qx");
      ok(tri_domain_download(d, TRI_FIELD_QY, bqy.data(), n), "download qy");
      if (!a.max_value_print_option.empty()) ok(tri_domain_download(d, TRI_FIELD_MAXH, bmh.data(), n), "download maxh");
      T.stop("compute");
      const int pid = c.print_id, itc = c.it_count;
      const double t_out = simtime, avg_dt = c.average_dt;
      writing = std::async(std::launch::async, [&out, &a, &bh, &bqx, &bqy, &bmh, pid, itc, t_out, avg_dt]() {
        const std::string& po = a.print_option;
        if (po.find('h') != std::string::npos) out.write("H", bh, pid);
        if (po.find('u') != std::string::npos) out.write("QX", bqx, pid);
        if (po.find('v') != std::string::npos) out.write("QY", bqy, pid);
        if (!a.max_value_print_option.empty() && a.max_value_print_option.find('h') != std::string::npos)
          out.write("MH", bmh, pid);
        std::cerr << C_BLUE "[" << pid << "]" C_RESET " File written at time " << t_out << " seconds.\n";
        out.restart_cfg(t_out, pid, avg_dt, itc);
        std::ofstream cid("cid");
        cid << pid;
      });
      T.stop("simulation");
      T.stop("total");
      out.times(T, c.print_id);
      T.start("simulation");
      T.start("total");
    }
    ok(tri_domain_set_clock(d, &c), "set clock");
    if ((p.events & TRI_EV_END) || (p.steps == 0 && p.events == 0)) break;
  }
  finish_writing();
  if (a.time_series_flag) observe();
  T.stop("simulation");
  T.stop("total");
  out.times(T, -1);
  std::cerr << C_GRAY "[INFO] " C_RESET " Time: " << simtime << "\tdt: "
            << (it_count_average ? c.average_dt / it_count_average : 0.0) << "\tit: " << c.it_count << std::endl;
  std::cerr << C_GREEN "[OK] " C_RESET "Simulation ends" << std::endl;
  return 0;
}

}  // namespace

// `triton_b200 --dump-problem <dir> <cfg>`: loads and preprocesses the case
// exactly as a run would, writes the padded arrays and tables as raw little
// endian files into <dir> and exits without touching a GPU (for tests).
int dump_problem(const char* argv0, const std::string& dir, const std::string& cfg) {
  Problem P = load_problem(argv0, cfg, 0);
  auto put = [&](const std::string& name, const void* p, size_t bytes) {
    std::ofstream f(dir + "/" + name, std::ios::binary);
    f.write(reinterpret_cast<const char*>(p), bytes);
  };
  auto putd = [&](const std::string& name, const std::vector<double>& v) { put(name, v.data(), v.size() * 8); };
  auto puti = [&](const std::string& name, const std::vector<int32_t>& v) { put(name, v.data(), v.size() * 4); };
  putd("h.f64", P.h);
  putd("qx.f64", P.qx);
  putd("qy.f64", P.qy);
  putd("z.f64", P.z);
  putd("n2.f64", P.n2);
  putd("maxh.f64", P.maxh);
  puti("src_cells.i32", P.src_cells);
  putd("hyg_t.f64", P.hyg_t);
  putd("hyg_v.f64", P.hyg_v);
  puti("zone.i32", P.zone);
  putd("roff_t.f64", P.roff_t);
  putd("roff_v.f64", P.roff_v);
  puti("bc_cells.i32", P.bc_cells);
  puti("bc_types.i32", P.bc_types);
  puti("bc_start.i32", P.bc_start);
  puti("bc_nrows.i32", P.bc_nrows);
  putd("bc_v1.f64", P.bc_v1);
  putd("bc_v2.f64", P.bc_v2);
  puti("obs_cells.i32", P.obs_cells);
  std::ofstream f(dir + "/info.txt");
  f << std::setprecision(17) << "rows " << P.rows << "\ncols " << P.cols << "\ndx " << P.dem.cell << "\nxll "
    << P.dem.xll << "\nyll " << P.dem.yll << "\ninit_dt " << P.init_dt << "\nrunoff_row " << P.runoff_row
    << "\nnroff " << P.nroff << "\nsimtime " << P.simtime << "\ncourant " << P.args.courant << "\nhextra "
    << P.args.hextra << "\n";
  // the loop parameters of triton_simulate.h (as the run sets its clock)
  const Args& a = P.args;
  f << "sim_duration " << a.sim_duration << "\nprint_interval " << a.print_interval << "\nprint_observation "
    << a.print_observation << "\ntime_series " << a.time_series_flag << "\nit_print " << a.it_print
    << "\nit_count " << a.it_count << "\ntime_increment_fixed " << a.time_increment_fixed << "\ntime_step "
    << a.time_step << "\nopen_boundaries " << a.open_boundaries << "\ncheckpoint_id " << a.checkpoint_id
    << "\nnzones " << P.nroff << "\nroff_rows " << P.roff_rows << "\nhyg_rows " << P.hyg_rows << "\n";
  return 0;
}

// `triton_b200 --format-fixed6 <in.f64> <out.txt>`: the ASCII raster text of
// raw little-endian doubles, one per line (for tests; no GPU).
int format_fixed6(const std::string& in, const std::string& outp) {
  std::ifstream f(in, std::ios::binary);
  std::vector<char> raw((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  std::string text;
  for (size_t i = 0; i + 8 <= raw.size(); i += 8) {
    double v;
    std::memcpy(&v, raw.data() + i, 8);
    trihost::append_fixed6(text, v);
    text.push_back('\n');
  }
  std::ofstream o(outp, std::ios::binary);
  o.write(text.data(), (std::streamsize)text.size());
  return 0;
}

int main(int argc, char** argv) {
  try {
    if (argc >= 4 && std::strcmp(argv[1], "--dump-problem") == 0) return dump_problem(argv[0], argv[2], argv[3]);
    if (argc >= 4 && std::strcmp(argv[1], "--format-fixed6") == 0) return format_fixed6(argv[2], argv[3]);
    return run(argc, argv);
  } catch (const InputError& e) {
    std::cerr << C_RED "[ERROR] " C_RESET << e.what() << std::endl;
    return EXIT_FAILURE;
  } catch (const std::exception& e) {
    std::cerr << C_RED "[ERROR] " C_RESET << e.what() << std::endl;
    return EXIT_FAILURE;
  }
}
