// On-disk formats through the C++ mirrors (pfc::b200::BinaryWriter, BinaryReader,
// VTKWriter, format_with_number): host only, no GPU.  Checks the byte layout of
// each file against the rules of the reference's writers.  Exit code 0 = pass.
#include <openpfc_b200/pfc_b200.hpp>

#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <iterator>
#include <sstream>

namespace b = pfc::b200;

static int failures = 0;
#define EXPECT(c)                                                   \
  do {                                                              \
    if (!(c)) {                                                     \
      std::cerr << __FILE__ << ":" << __LINE__ << ": " #c << "\n"; \
      ++failures;                                                   \
    }                                                               \
  } while (0)

static std::string slurp(const std::string &fn) {
  std::ifstream f(fn, std::ios::binary);
  return std::string(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
}

int main(int argc, char **argv) {
  const std::string dir = argc > 1 ? argv[1] : ".";
  // format_with_number (frontend/utils/utils.hpp:96-139)
  EXPECT(b::format_with_number("output_%d.dat", 3) == "output_3.dat");
  EXPECT(b::format_with_number("frame_%04d.vti", 7) == "frame_0007.vti");
  EXPECT(b::format_with_number("result_%-5d.bin", 1) == "result_1    .bin");
  EXPECT(b::format_with_number("plain.bin", 9) == "plain.bin");
  for (const char *bad : {"a_%s.bin", "a_%d_%d.bin", "a_%n", "a_%f.bin", "%"}) {
    bool threw = false;
    try {
      b::format_with_number(bad, 1);
    } catch (const std::invalid_argument &) {
      threw = true;
    }
    EXPECT(threw);
  }

  // BinaryWriter / BinaryReader: whole grid, x fastest, raw doubles
  const std::array<int, 3> g{5, 4, 3};
  std::vector<double> a(60);
  for (size_t i = 0; i < a.size(); ++i) a[i] = 0.25 * (double)i - 3.0;
  b::BinaryWriter w(dir + "/psi_%02d.bin");
  w.set_domain(g, g, {0, 0, 0});
  w.write(4, a);
  const std::string raw = slurp(dir + "/psi_04.bin");
  EXPECT(raw.size() == 60 * sizeof(double));
  EXPECT(std::memcmp(raw.data(), a.data(), raw.size()) == 0);
  std::vector<double> back(60, 0.0);
  b::BinaryReader r;
  r.set_domain(g, g, {0, 0, 0});
  r.read(dir + "/psi_04.bin", back);
  EXPECT(back == a);
  // a sub-box lands at its place in the global array (file truncated first)
  std::vector<double> sub(2 * 3 * 2);
  for (size_t i = 0; i < sub.size(); ++i) sub[i] = 100.0 + (double)i;
  b::BinaryWriter ws(dir + "/sub.bin");
  ws.set_domain(g, {2, 3, 2}, {1, 1, 1});
  ws.write(0, sub);
  std::vector<double> box(12, 0.0);
  b::BinaryReader rs;
  rs.set_domain(g, {2, 3, 2}, {1, 1, 1});
  rs.read(dir + "/sub.bin", box);
  EXPECT(box == sub);
  const std::string sraw = slurp(dir + "/sub.bin");
  double first;
  std::memcpy(&first, sraw.data() + sizeof(double) * ((1 * 4 + 1) * 5 + 1), sizeof first);
  EXPECT(first == 100.0);
  // complex: interleaved re, im
  std::vector<std::complex<double>> c(60);
  for (size_t i = 0; i < c.size(); ++i) c[i] = {(double)i, -(double)i};
  b::BinaryWriter wc(dir + "/hat.bin");
  wc.set_domain(g, g, {0, 0, 0});
  wc.write(0, c);
  EXPECT(slurp(dir + "/hat.bin") == std::string(reinterpret_cast<const char *>(c.data()), 120 * sizeof(double)));
  // size contract
  bool threw = false;
  try {
    std::vector<double> wrong(7);
    w.write(0, wrong);
  } catch (const std::runtime_error &) {
    threw = true;
  }
  EXPECT(threw);
  threw = false;
  try {
    std::vector<double> big(60);
    b::BinaryReader rr;
    rr.set_domain({6, 4, 3}, {6, 4, 3}, {0, 0, 0});
    big.resize(72);
    rr.read(dir + "/psi_04.bin", big);  // file holds 60 values
  } catch (const std::exception &) {
    threw = true;
  }
  EXPECT(threw);

  // VTKWriter (src/openpfc/frontend/io/vtk_writer.cpp:70-108,166-225)
  b::VTKWriter v(dir + "/f_%d.vti");
  v.set_domain(g, g, {0, 0, 0});
  v.set_origin({-1.5, 0, 2});
  v.set_spacing({0.785398163397448, 1, 0.5});
  v.set_field_name("density");
  v.write(2, a);
  const std::string vti = slurp(dir + "/f_2.vti");
  std::ostringstream head;
  head << "<?xml version=\"1.0\" encoding=\"utf-8\"?>\n"
       << "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n"
       << "  <ImageData WholeExtent=\"0 4 0 3 0 2\" Origin=\"-1.5 0 2\" Spacing=\"0.785398 1 0.5\">\n"
       << "    <Piece Extent=\"0 4 0 3 0 2\">\n"
       << "      <PointData>\n"
       << "        <DataArray type=\"Float64\" Name=\"density\" NumberOfComponents=\"1\" format=\"appended\" offset=\"0\"/>\n"
       << "      </PointData>\n"
       << "    </Piece>\n"
       << "  </ImageData>\n"
       << "  <AppendedData encoding=\"raw\">\n"
       << "_";
  const std::string h = head.str();
  EXPECT(vti.compare(0, h.size(), h) == 0);
  std::uint64_t nbytes = 0;
  std::memcpy(&nbytes, vti.data() + h.size(), 8);
  EXPECT(nbytes == 60 * sizeof(double));
  EXPECT(std::memcmp(vti.data() + h.size() + 8, a.data(), 60 * sizeof(double)) == 0);
  EXPECT(vti.substr(h.size() + 8 + 60 * sizeof(double)) == "\n  </AppendedData>\n</VTKFile>\n");

  std::cout << (failures ? "FAIL " : "ok ") << failures << "\n";
  return failures ? 1 : 0;
}
