// Sample driver with the reference sample's command line and output
// (r-ccs-cms/sbd samples/selected_basis_diagonalization/main.cc:17-226),
// running sbd::tpb::diag on one B200 through libsbdgpu.so.
#include <fstream>
#include <iostream>

#include "sbd/sbd.h"

int main(int argc, char* argv[]) {
#ifdef SBD_GPU_HAVE_MPI
  int provided;
  MPI_Init_thread(&argc, &argv, MPI_THREAD_FUNNELED, &provided);
  MPI_Comm comm = MPI_COMM_WORLD;
#else
  MPI_Comm comm = 0;
#endif
  auto sbd_data = sbd::tpb::generate_sbd_data(argc, argv);
  std::string adetfile("alphadets.txt"), fcidumpfile("fcidump.txt"), loadname, savename, carryoverfile;
  for (int i = 0; i + 1 < argc; i++) {
    std::string a(argv[i]);
    if (a == "--adetfile") adetfile = argv[++i];
    else if (a == "--fcidump") fcidumpfile = argv[++i];
    else if (a == "--loadname") loadname = argv[++i];
    else if (a == "--savename") savename = argv[++i];
    else if (a == "--carryoverfile") carryoverfile = argv[++i];
  }
  double energy = 0.0;
  std::vector<double> density;
  std::vector<std::vector<size_t>> cobits;
  std::vector<std::vector<double>> one_p_rdm, two_p_rdm;
  std::cout.precision(16);
  try {
    sbd::FCIDump fcidump = sbd::LoadFCIDump(fcidumpfile);
    int L = 0;
    for (const auto& [key, value] : fcidump.header) {
      if (key == "NORB") L = std::atoi(value.c_str());
    }
    std::vector<std::vector<size_t>> adet, bdet;
    sbd::LoadAlphaDets(adetfile, adet, sbd_data.bit_length, L);
    bdet = adet;
    if (sbd_data.do_shuffle != 0) {
      sbd::ShuffleDet(adet, 1729u);
      sbd::ShuffleDet(bdet, 137u);
    }
    sbd::tpb::diag(comm, sbd_data, fcidump, adet, bdet, loadname, savename, energy, density, cobits, one_p_rdm,
                   two_p_rdm);
    std::cout << " Sample-based diagonalization: Energy = " << energy << std::endl;
    std::cout << " Sample-based diagonalization: density = ";
    for (size_t i = 0; i < density.size() / 2; i++)
      std::cout << ((i == 0) ? "[" : ",") << density[2 * i] + density[2 * i + 1];
    std::cout << std::endl;
    std::cout << " Sample-based diagonalization: carryover bitstrings = ";
    for (size_t i = 0; i < std::min(cobits.size(), (size_t)6); i++)
      std::cout << " " << sbd::makestring(cobits[i], sbd_data.bit_length, L);
    if (cobits.size() > 6) std::cout << " ... " << sbd::makestring(cobits.back(), sbd_data.bit_length, L);
    std::cout << std::endl;
    if (!carryoverfile.empty()) {
      std::ofstream o(carryoverfile);
      for (auto& c : cobits) o << sbd::makestring(c, sbd_data.bit_length, L) << std::endl;
    }
    if (!one_p_rdm.empty()) {
      auto ints = sbd::gpu_detail::setup_integrals(fcidump);
      auto I2 = [&](int p, int q, int r, int s) {
        auto pr = [](int i, int j) { int a = std::max(i, j), b = std::min(i, j); return (size_t)a * (a + 1) / 2 + b; };
        size_t ij = pr(p, q), kl = pr(r, s), a = std::max(ij, kl), b = std::min(ij, kl);
        return ints.eri[a * (a + 1) / 2 + b];
      };
      double onebody = 0.0, twobody = 0.0;
      std::ofstream o1("1pRDM.txt");
      o1.precision(16);
      for (int io = 0; io < L; io++)
        for (int jo = 0; jo < L; jo++) {
          double v = one_p_rdm[0][io + L * jo] + one_p_rdm[1][io + L * jo];
          o1 << io << " " << jo << " " << v << std::endl;
          onebody += ints.h1[(size_t)io * L + jo] * v;
        }
      std::ofstream o2("2pRDM.txt");
      o2.precision(16);
      size_t L2 = (size_t)L * L;
      for (int io = 0; io < L; io++)
        for (int jo = 0; jo < L; jo++)
          for (int ia = 0; ia < L; ia++)
            for (int ja = 0; ja < L; ja++) {
              size_t k = io + L * jo + L2 * (ia + (size_t)L * ja);
              double v = two_p_rdm[0][k] + two_p_rdm[1][k] + two_p_rdm[2][k] + two_p_rdm[3][k];
              o2 << io << " " << jo << " " << ia << " " << ja << " " << v << std::endl;
              twobody += 0.5 * I2(io, ia, jo, ja) * v;
            }
      std::cout << " One-Body energy = " << onebody << std::endl;
      std::cout << " Two-Body energy = " << twobody << std::endl;
      std::cout << " One-Body + Two-Body energy = " << onebody + twobody << std::endl;
    }
  } catch (const std::exception& e) {
    std::cerr << "diag: " << e.what() << std::endl;
    return 1;
  }
  return 0;
}
