// `poisson-recon`: the command-line front end of the library, a drop-in for the crate's binary
// (src/main.rs:7-50): the same flags, defaults, messages and exit codes, calling the C ABI
// (pr_ply_read_points -> pr_reconstruct -> pr_ply_write_mesh).
//
//   poisson-recon -i points.ply [-o output.ply] [-d 8] [--samples-per-node 1.5]
//                 [--cg-accuracy 0.001] [--cg-iters 500] [--point-weight 0.0] [--scale 1.1] [-v]
//
// Extensions (not in the crate): --solve-mode converged|reference (default converged: the
// crate's fine system solved to --target-rel-residual; "reference" runs the crate's cascade
// schedule), --precision mixed|fp64, --target-rel-residual R, --degree 1|2 (quadratic B-spline
// node functions), --binary (binary PLY output), --device N.
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "poisson_recon.h"

namespace {

const char* kUsage = "Usage: poisson-recon [OPTIONS] --input <INPUT>";

void usage_error(const std::string& msg) {
  std::fprintf(stderr, "error: %s\n\n%s\n\nFor more information, try '--help'.\n", msg.c_str(), kUsage);
  std::exit(2);
}

void print_help() {
  std::printf(
      "Screened Poisson Surface Reconstruction\n\n%s\n\n"
      "Options:\n"
      "  -i, --input <INPUT>                      oriented points (PLY with x y z nx ny nz)\n"
      "  -o, --output <OUTPUT>                    mesh file [default: output.ply]\n"
      "  -d, --depth <DEPTH>                      grid depth, res = 2^depth (1..10) [default: 8]\n"
      "      --samples-per-node <SAMPLES_PER_NODE>  accepted, unused [default: 1.5]\n"
      "      --cg-accuracy <CG_ACCURACY>          reference schedule: CG accuracy [default: 0.001]\n"
      "      --cg-iters <CG_ITERS>                reference schedule: CG iterations [default: 500]\n"
      "      --point-weight <POINT_WEIGHT>        screening weight [default: 0.0]\n"
      "      --scale <SCALE>                      bounding-box scale [default: 1.1]\n"
      "  -v, --verbose                            print counts and stage timings\n"
      "      --solve-mode <converged|reference>   solver (default converged)\n"
      "      --precision <mixed|fp64>             converged mode arithmetic [default: mixed]\n"
      "      --target-rel-residual <R>            converged mode target [default: 1e-6]\n"
      "      --degree <1|2>                       B-spline degree of the node functions [default: 1]\n"
      "      --binary                             write binary_little_endian PLY\n"
      "      --device <N>                         CUDA device [default: 0]\n"
      "  -h, --help                               Print help\n"
      "  -V, --version                            Print version\n",
      kUsage);
}

template <typename T>
T parse_num(const std::string& flag, const std::string& v);
template <>
double parse_num<double>(const std::string& flag, const std::string& v) {
  char* end = nullptr;
  errno = 0;
  const double x = std::strtod(v.c_str(), &end);
  if (v.empty() || *end != '\0') usage_error("invalid value '" + v + "' for '" + flag + "': invalid float literal");
  return x;
}
template <>
unsigned long long parse_num<unsigned long long>(const std::string& flag, const std::string& v) {
  char* end = nullptr;
  errno = 0;
  const unsigned long long x = std::strtoull(v.c_str(), &end, 10);
  if (v.empty() || *end != '\0' || v[0] == '-' || errno == ERANGE)
    usage_error("invalid value '" + v + "' for '" + flag + "': invalid digit found in string");
  return x;
}

struct Args {
  std::string input, output = "output.ply";
  unsigned long long depth = 8, cg_iters = 500, device = 0;
  double samples_per_node = 1.5, cg_accuracy = 0.001, point_weight = 0.0, scale = 1.1;
  bool verbose = false, binary = false, have_input = false;
  int solve_mode = PR_SOLVE_CONVERGED, precision = PR_PRECISION_MIXED;
  double target = 1e-6;
  unsigned degree = 1;
};

Args parse(int argc, char** argv) {
  Args a;
  for (int i = 1; i < argc; ++i) {
    std::string arg = argv[i], val;
    bool has_val = false;
    std::string name;
    if (arg.rfind("--", 0) == 0) {
      const size_t eq = arg.find('=');
      name = arg.substr(2, eq == std::string::npos ? std::string::npos : eq - 2);
      if (eq != std::string::npos) {
        val = arg.substr(eq + 1);
        has_val = true;
      }
    } else if (arg.size() >= 2 && arg[0] == '-') {
      const char c = arg[1];
      static const char* shorts[][2] = {{"i", "input"}, {"o", "output"}, {"d", "depth"}, {"v", "verbose"},
                                        {"h", "help"}, {"V", "version"}};
      for (auto& s : shorts)
        if (c == s[0][0]) name = s[1];
      if (name.empty()) usage_error("unexpected argument '" + arg + "' found");
      if (arg.size() > 2) {
        val = arg.substr(arg[2] == '=' ? 3 : 2);
        has_val = true;
      }
    } else {
      usage_error("unexpected argument '" + arg + "' found");
    }
    auto need = [&]() -> std::string {
      if (has_val) return val;
      if (i + 1 >= argc) usage_error("a value is required for '--" + name + " <" + name + ">' but none was supplied");
      return argv[++i];
    };
    const std::string flag = "--" + name;
    if (name == "help") {
      print_help();
      std::exit(0);
    } else if (name == "version") {
      std::printf("poisson-recon 0.1.0\n");
      std::exit(0);
    } else if (name == "input") {
      a.input = need();
      a.have_input = true;
    } else if (name == "output") {
      a.output = need();
    } else if (name == "depth") {
      a.depth = parse_num<unsigned long long>(flag, need());
    } else if (name == "samples-per-node") {
      a.samples_per_node = parse_num<double>(flag, need());
    } else if (name == "cg-accuracy") {
      a.cg_accuracy = parse_num<double>(flag, need());
    } else if (name == "cg-iters") {
      a.cg_iters = parse_num<unsigned long long>(flag, need());
    } else if (name == "point-weight") {
      a.point_weight = parse_num<double>(flag, need());
    } else if (name == "scale") {
      a.scale = parse_num<double>(flag, need());
    } else if (name == "verbose") {
      if (has_val) usage_error("unexpected value '" + val + "' for '--verbose' found");
      a.verbose = true;
    } else if (name == "binary") {
      a.binary = true;
    } else if (name == "device") {
      a.device = parse_num<unsigned long long>(flag, need());
    } else if (name == "target-rel-residual") {
      a.target = parse_num<double>(flag, need());
    } else if (name == "solve-mode") {
      const std::string v = need();
      if (v == "converged") a.solve_mode = PR_SOLVE_CONVERGED;
      else if (v == "reference") a.solve_mode = PR_SOLVE_REFERENCE_SCHEDULE;
      else usage_error("invalid value '" + v + "' for '--solve-mode'");
    } else if (name == "degree") {
      const std::string v = need();
      if (v == "1") a.degree = 1;
      else if (v == "2") a.degree = 2;
      else usage_error("invalid value '" + v + "' for '--degree'");
    } else if (name == "precision") {
      const std::string v = need();
      if (v == "mixed") a.precision = PR_PRECISION_MIXED;
      else if (v == "fp64") a.precision = PR_PRECISION_FP64;
      else usage_error("invalid value '" + v + "' for '--precision'");
    } else {
      usage_error("unexpected argument '" + arg + "' found");
    }
  }
  if (!a.have_input) usage_error("the following required arguments were not provided:\n  --input <INPUT>");
  return a;
}

}  // namespace

int main(int argc, char** argv) {
  const Args a = parse(argc, argv);
  double* pts = nullptr;
  uint64_t n = 0;
  if (pr_ply_read_points(a.input.c_str(), &pts, &n) != PR_OK) {
    std::fprintf(stderr, "Error: %s\n", pr_last_error());
    return 1;
  }
  if (n == 0) {
    std::fprintf(stderr, "No points found.\n");
    return 1;
  }
  if (a.verbose) std::fprintf(stderr, "Read %llu oriented points\n", (unsigned long long)n);

  pr_params p = pr_params_default();
  p.depth = a.depth > 0xffffffffull ? 0xffffffffu : (uint32_t)a.depth;
  p.samples_per_node = a.samples_per_node;
  p.scale = a.scale;
  p.cg_accuracy = a.cg_accuracy;
  p.cg_iters = a.cg_iters;
  p.point_weight = a.point_weight;
  p.verbose = 0;  // the crate's library prints nothing; the timing lines below are the CLI's
  p.solve_mode = a.solve_mode;
  p.precision = a.precision;
  p.target_rel_residual = a.target;
  p.degree = a.degree;

  pr_context* ctx = nullptr;
  pr_mesh mesh;
  pr_stats st;
  std::memset(&mesh, 0, sizeof(mesh));
  int rc = pr_context_create((int)a.device, nullptr, &ctx);
  if (rc == PR_OK) rc = pr_ctx_reconstruct(ctx, pts, n, &p, &mesh, &st);
  pr_host_free(pts);
  if (rc != PR_OK) {
    std::fprintf(stderr, "Error: %s\n", pr_last_error());
    pr_context_destroy(ctx);
    return 1;
  }
  if (a.verbose) {
    std::fprintf(stderr, "Timing [s]: xform=%.3f tree=%.3f sys=%.3f solve=%.3f extract=%.3f total=%.3f\n",
                 st.time_transform, st.time_tree, st.time_system, st.time_solve, st.time_extract, st.time_total);
    std::fprintf(stderr, "FEM nodes=%llu, matrix NNZ=%llu\n", (unsigned long long)st.fem_nodes,
                 (unsigned long long)st.matrix_nnz);
    std::fprintf(stderr, "Mesh: %llu verts, %llu tris, iso=%.6f\n", (unsigned long long)st.mesh_vertices,
                 (unsigned long long)st.mesh_triangles, st.iso_value);
  }
  rc = pr_ply_write_mesh(a.output.c_str(), &mesh, a.binary ? PR_PLY_BINARY : PR_PLY_ASCII);
  pr_mesh_free(&mesh);
  pr_context_destroy(ctx);
  if (rc != PR_OK) {
    std::fprintf(stderr, "Error writing: %s\n", pr_last_error());
    return 1;
  }
  if (a.verbose) std::fprintf(stderr, "Wrote %s\n", a.output.c_str());
  return 0;
}
