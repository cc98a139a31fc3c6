// Reference-side codec harness (test infrastructure).  Compiled by
// oracle/Makefile against the reference's own topo_opt/fem_interface.h and
// topo_opt/serialization.h, used in their standalone (non-Taichi) mode
// (fem_interface.h:28-36).  It writes the golden blobs and dumps blobs written by
// other codecs as text, so the wire format is pinned by the reference's own code.
//
//   codec_harness kat <inputs.bin> <outputs.bin>   write the known-answer blobs
//   codec_harness dump-in <file>                   print an FEMInputs blob
//   codec_harness dump-out <file>                  print an FEMOutputs blob
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "fem_interface.h"

using namespace fem_interface;

// Values of the reference's interface test (topo_opt/interface_test.cpp:45-166),
// with the grid shrunk from 128x256x512 to 16x32x64 to keep the fixture small.
static void fill_kat(FEMInputs& param) {
  param.version_major = FEM_INTERFACE_VERSION_MAJOR;
  param.version_minor = FEM_INTERFACE_VERSION_MINOR;
  param.resolution[0] = 16;
  param.resolution[1] = 32;
  param.resolution[2] = 64;
  param.use_density_only = true;
  param.dx = 0.01f;
  for (int i = 0; i < 17; i++) {
    ForceOnNode f;
    f.coord[0] = i * 2 + 1;
    f.coord[1] = i * i + 14;
    f.coord[2] = i / 3 + 1;
    f.f[0] = std::sqrt(1.0 * i);
    f.f[1] = i * i;
    f.f[2] = i * i * i / 10000.0;
    param.forces.push_back(f);
  }
  DirichletOnNode d;
  d.coord[0] = 95; d.coord[1] = 6; d.coord[2] = 3; d.axis = 2; d.value = 0.1234;
  param.dirichlet_nodes.push_back(d);
  d.coord[0] = 94; d.coord[1] = 11; d.coord[2] = 16; d.axis = 1; d.value = 0.5432;
  param.dirichlet_nodes.push_back(d);
  param.krylov.tolerance = 1e-5;
  param.krylov.max_iterations = 10000;
  param.krylov.restart_iterations = 1000;
  param.krylov.print_residuals = true;
  param.caller_method = "topology_optimization";
  param.extra_ints["multigrid_num_pre_smoothing"] = 2;
  param.extra_ints["multigrid_num_post_smoothing"] = 3;
  param.extra_strings["log_file_path"] = "/tmp/fem_solver.log";
  param.extra_doubles["smoother_jacobi_damping"] = 0.66667f;
  param.global_mu = 2.0f;
  param.global_lambda = 1.0f;
  param.mg_level = 5;
  param.explicit_mg_level = 2;
  param.pre_and_post_smoothing_iter = 1;
  param.bottom_smoothing_iter = 600;
  param.jacobi_damping = 0.4;
  int centers[3];
  for (int i = 0; i < 3; i++) centers[i] = param.resolution[i] / 2;
  const int depth = 6;
  auto node_inside = [&](int* c) {
    for (int i = 0; i < 3; i++)
      if (centers[i] - depth < c[i] && c[i] < centers[i] + depth) return true;
    return false;
  };
  auto cell_inside = [&](int* c) {
    for (int i = 0; i < 3; i++)
      if (centers[i] - depth < c[i] && c[i] < centers[i] + depth - 1) return true;
    return false;
  };
  param.density.resolution[0] = param.resolution[0];
  param.density.resolution[1] = param.resolution[1];
  param.density.resolution[2] = param.resolution[2];
  for (int i = 0; i < param.resolution[0]; i += 4)
    for (int j = 0; j < param.resolution[1]; j += 4)
      for (int k = 0; k < param.resolution[2]; k += 4) {
        bool active = false;
        for (int ii = 0; ii < 4; ii++)
          for (int jj = 0; jj < 4; jj++)
            for (int kk = 0; kk < 4; kk++) {
              int c[3] = {i + ii, j + jj, k + kk};
              if (node_inside(c)) active = true;
            }
        if (!active) continue;
        FEMInputs::ScalarGrid::Block block;
        block.base_coordinates[0] = i;
        block.base_coordinates[1] = j;
        block.base_coordinates[2] = k;
        block.reset_data();
        for (int ii = 0; ii < 4; ii++)
          for (int jj = 0; jj < 4; jj++)
            for (int kk = 0; kk < 4; kk++) {
              int c[3] = {i + ii, j + jj, k + kk};
              if (cell_inside(c)) block.get(ii, jj, kk) = i * jj + k - j + kk * ii;
            }
        param.density.blocks.push_back(block);
      }
  param.set_solver_state_ptr((void*)(0x1234567890543200ul));
}

static void write_file(const std::string& fn, const std::vector<uint8_t>& data, size_t n) {
  std::ofstream f(fn, std::ios::binary);
  f.write(reinterpret_cast<const char*>(data.data()), n);
}

static std::vector<uint8_t> read_file(const std::string& fn) {
  std::ifstream f(fn, std::ios::binary);
  return std::vector<uint8_t>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

template <typename M>
static void print_map(const char* name, const M& m) {
  std::printf("%s %zu\n", name, m.size());
  for (auto& kv : m) std::printf("  %s = %s\n", kv.first.c_str(), std::to_string(kv.second).c_str());
}

static void print_base(const FEMDataBase& p) {
  std::printf("version %d %d\n", p.version_major, p.version_minor);
  std::printf("extra_strings %zu\n", p.extra_strings.size());
  for (auto& kv : p.extra_strings) std::printf("  %s = %s\n", kv.first.c_str(), kv.second.c_str());
  std::printf("extra_ints %zu\n", p.extra_ints.size());
  for (auto& kv : p.extra_ints) std::printf("  %s = %d\n", kv.first.c_str(), kv.second);
  std::printf("extra_doubles %zu\n", p.extra_doubles.size());
  for (auto& kv : p.extra_doubles) std::printf("  %s = %.17g\n", kv.first.c_str(), kv.second);
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  std::string cmd = argv[1];
  if (cmd == "kat" && argc >= 4) {
    FEMInputs param;
    fill_kat(param);
    param.preserved_buffer_size = (1u << 20) + param.density.blocks.size() * sizeof(FEMOutputs::VectorGrid::Block);
    BinaryOutputSerializer ser;
    ser.initialize();
    param.io(ser);
    ser.finalize();
    write_file(argv[2], ser.data, ser.head);
    // outputs of the fake solver of interface_test.cpp:7-34 (displacement = density + p)
    FEMOutputs out;
    out.displacements.resolution[0] = param.resolution[0];
    out.displacements.resolution[1] = param.resolution[1];
    out.displacements.resolution[2] = param.resolution[2];
    out.residual_field.resolution[0] = out.residual_field.resolution[1] = out.residual_field.resolution[2] = 0;
    for (auto& db : param.density.blocks) {
      FEMOutputs::VectorGrid::Block b;
      for (int i = 0; i < 3; i++) b.base_coordinates[i] = db.base_coordinates[i];
      for (int e = 0; e < 64; e++) {
        for (int p = 0; p < 3; p++) b.data[e][p] = db.data[e] + p;
        b.data[e][3] = 0.5 * e;
      }
      out.displacements.blocks.push_back(b);
    }
    out.info = "known-answer outputs";
    out.residuals = {1.0, 0.25, 1e-5};
    out.error_code = 7;
    out.success = true;
    out.extra_ints["iterations"] = 3;
    BinaryOutputSerializer so;
    so.initialize();
    so("outputs", out);
    so.finalize();
    write_file(argv[3], so.data, so.head);
    return 0;
  }
  if (cmd == "dump-in") {
    auto data = read_file(argv[2]);
    FEMInputs p;
    BinaryInputSerializer ser;
    ser.initialize(data.data());
    p.io(ser);
    ser.finalize();
    print_base(p);
    std::printf("dx %.17g preserved %zu use_density_only %d\n", p.dx, p.preserved_buffer_size, int(p.use_density_only));
    std::printf("global %.17g %.17g\n", p.global_mu, p.global_lambda);
    std::printf("density res %d %d %d blocks %zu\n", p.density.resolution[0], p.density.resolution[1],
                p.density.resolution[2], p.density.blocks.size());
    double checksum = 0;
    long basesum = 0;
    for (auto& b : p.density.blocks) {
      basesum += b.base_coordinates[0] * 1000003L + b.base_coordinates[1] * 1009L + b.base_coordinates[2];
      for (int e = 0; e < 64; e++) checksum += b.data[e] * (1 + e % 7);
    }
    std::printf("density basesum %ld checksum %.17g\n", basesum, checksum);
    std::printf("mg %d %d %d %d %.17g\n", p.mg_level, p.explicit_mg_level, p.pre_and_post_smoothing_iter,
                p.bottom_smoothing_iter, p.jacobi_damping);
    std::printf("resolution %d %d %d\n", p.resolution[0], p.resolution[1], p.resolution[2]);
    std::printf("forces %zu\n", p.forces.size());
    for (auto& f : p.forces)
      std::printf("  %d %d %d %.17g %.17g %.17g\n", f.coord[0], f.coord[1], f.coord[2], f.f[0], f.f[1], f.f[2]);
    std::printf("dirichlet_nodes %zu\n", p.dirichlet_nodes.size());
    for (auto& d : p.dirichlet_nodes)
      std::printf("  %d %d %d %d %.17g\n", d.coord[0], d.coord[1], d.coord[2], d.axis, d.value);
    std::printf("dirichlet_cells %zu\n", p.dirichlet_cells.size());
    std::printf("krylov %.17g %d %d %d\n", p.krylov.tolerance, p.krylov.max_iterations, p.krylov.restart_iterations,
                int(p.krylov.print_residuals));
    std::printf("caller %s\n", p.caller_method.c_str());
    std::printf("state_ptr %p\n", p.get_solver_state_ptr());
    return 0;
  }
  if (cmd == "dump-out") {
    auto data = read_file(argv[2]);
    FEMOutputs o;
    BinaryInputSerializer ser;
    ser.initialize(data.data());
    ser("outputs", o);
    ser.finalize();
    print_base(o);
    std::printf("displacements res %d %d %d blocks %zu\n", o.displacements.resolution[0], o.displacements.resolution[1],
                o.displacements.resolution[2], o.displacements.blocks.size());
    double checksum = 0;
    for (auto& b : o.displacements.blocks)
      for (int e = 0; e < 64; e++)
        for (int p = 0; p < 4; p++) checksum += b.data[e][p] * (1 + (e + p) % 5);
    std::printf("displacements checksum %.17g\n", checksum);
    std::printf("residual_field blocks %zu\n", o.residual_field.blocks.size());
    std::printf("info %s\n", o.info.c_str());
    std::printf("residuals %zu\n", o.residuals.size());
    for (double r : o.residuals) std::printf("  %.17g\n", r);
    std::printf("error_code %d success %d\n", o.error_code, int(o.success));
    return 0;
  }
  return 2;
}
