// tri_host.h -- the C++ drop-in host around the C ABI: configuration,
// input rasters and forcing tables, preprocessing, the time loop and the
// output files of the reference executable (triton.exe), for one rank.
#pragma once

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace trihost {

// An input problem the reference would also reject: the message is printed
// the way the reference prints it and the executable exits with failure.
struct InputError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// The cfg keys of ConfigUtils::arguments (config_utils.h:27-100), parsed with
// the same defaults and conversions (config_utils.h:422-517).
struct Args {
  bool time_increment_fixed = false, time_series_flag = false, gpu_direct_flag = false, open_boundaries = false;
  int checkpoint_id = 0, num_sources = 0, num_runoffs = 0, num_extbc = 0, it_count = 0, it_print = 10000;
  int factor_interval_domain_decomposition = 0;
  double time_step = 0, sim_start_time = 0, sim_duration = 0, print_interval = 0, print_observation = 0;
  double courant = 0, const_mann = 0, hextra = 0;
  std::string outfile_pattern, hydrograph_filename, runoff_filename, print_option, max_value_print_option;
  std::string input_format, input_option, output_format, output_option, projection, dem_filename;
  std::string header_filename, src_loc_file, runoff_map, observation_loc_file, extbc_file, extbc_dir;
  std::string h_infile, qx_infile, qy_infile, n_infile, input_folder, output_folder, domain_decomposition;
  std::vector<double> src_x, src_y, obs_x, obs_y, ebc_x1, ebc_y1, ebc_x2, ebc_y2;
  std::vector<int> ebc_type;
  std::vector<std::string> ebc_fname;
};

std::map<std::string, std::string> parse_cfg(const std::string& content);
Args get_args(const std::string& cfg_content);
std::string read_file(const std::string& path);
std::string root_dir(const char* argv0);
std::vector<std::string> split(const std::string& s, char delim);
std::string trim(std::string s);

// Rasters, row-major.
struct DemHeader {
  int ncols = 0, nrows = 0;
  double xll = 0, yll = 0, cell = 0;
  int nodata = 0;
};
DemHeader read_dem_header(const std::string& path, bool ascii);
std::vector<double> read_dem(const std::string& path, int rows, int cols, bool ascii);
std::vector<double> read_raster(const std::string& path, int rows, int cols, bool ascii);
std::vector<int32_t> read_raster_int(const std::string& path, int rows, int cols, bool ascii);

// Comma tables with '%' comments (hydrograph, runoff, extbc type-1 series).
std::vector<std::vector<double>> read_table(const std::string& path);

// The preprocessed single-rank problem (what triton_init.h hands the device).
struct Problem {
  Args args;
  std::string cfg_content, project_dir;
  DemHeader dem;
  int rows = 0, cols = 0;  // padded
  std::vector<double> h, qx, qy, z, n2, maxh;
  // forcing (flattened as in triton_init.h)
  int nsrc = 0, hyg_rows = 0;
  std::vector<int32_t> src_cells;
  std::vector<double> hyg_t, hyg_v;
  int nroff = 0, roff_rows = 0, runoff_row = 0;
  std::vector<int32_t> zone;
  std::vector<double> roff_t, roff_v;
  std::vector<int32_t> bc_cells, bc_types, bc_start, bc_nrows;
  std::vector<double> bc_v1, bc_v2;
  std::vector<int32_t> obs_cells;
  double init_dt = 0, simtime = 0;
};

// triton<T>::triton + initialize (triton_init.h:11-81), single rank, SEQ input.
Problem load_problem(const std::string& argv0, const std::string& cfg_arg, int checkpoint_id);

}  // namespace trihost
