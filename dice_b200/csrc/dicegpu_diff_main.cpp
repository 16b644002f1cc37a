// dicegpu_diff -- compares two DICe text result files with DICe_Diff's
// command line (tools/DICe_Diff.cpp): dicegpu_diff <fileA> <fileB> [-t <tol>]
// [-f <floor>] [-v] [-n] [-p <count>].  Prints "End Result: TEST PASSED" and
// exits 0, or "End Result: TEST FAILED" and exits 1.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "dicegpu_results.h"

int main(int argc, char** argv) {
  if (argc == 2 && std::strcmp(argv[1], "-h") == 0) {
    std::printf(" dicegpu_diff (compares two DICe output files, numerical and string values)\n"
                " Syntax: dicegpu_diff <fileA> <fileB> [options]\n"
                " Options: -h show help message\n"
                "          -v verbose\n"
                "          -t <tol> relative tolerance\n"
                "          -f <value> floor, values below the floor in the gold file will not be tested\n"
                "          -n numerical values only\n"
                "          -p <count> parallel output number of processors\n");
    return 0;
  }
  if (argc < 3) {
    std::printf("You must provide two files to compare\n");
    return 1;
  }
  double tol = 1.0e-6, floor = 0.0;
  int use_floor = 0, numerical = 0, procs = 1, verbose = 0;
  for (int i = 3; i < argc; ++i) {
    if (std::strcmp(argv[i], "-v") == 0) verbose = 1;
    else if (std::strcmp(argv[i], "-n") == 0) numerical = 1;
    else if (std::strcmp(argv[i], "-t") == 0 && i + 1 < argc) tol = std::strtod(argv[++i], nullptr);
    else if (std::strcmp(argv[i], "-f") == 0 && i + 1 < argc) { floor = std::strtod(argv[++i], nullptr); use_floor = 1; }
    else if (std::strcmp(argv[i], "-p") == 0 && i + 1 < argc) procs = (int)std::strtol(argv[++i], nullptr, 0);
    else {
      std::fprintf(stderr, "Error, unrecognized option %s\n", argv[i]);
      return 2;
    }
  }
  std::vector<char> report(1 << 20);
  int failed = 0;
  const int rc = dicegpu_diff_files(argv[1], argv[2], tol, floor, use_floor, numerical, procs, &failed,
                                    report.data(), report.size());
  if (rc != 0) {
    std::printf("Error, could not read the files (%d)\nEnd Result: TEST FAILED\n", rc);
    return 1;
  }
  if (verbose) {
    std::printf("File A:                %s\nFile B (or base name): %s\nRelative Tol:          %g\n"
                "Floor value:           %g active %d\nNumber of processors:  %d\n%s",
                argv[1], argv[2], tol, floor, use_floor, procs, report.data());
  }
  std::printf(failed ? "End Result: TEST FAILED\n" : "End Result: TEST PASSED\n");
  return failed ? 1 : 0;
}
