// Drop-in for the reference's entry point (src/main.cpp:12-20): read the ConfigFile, build the
// Simulation, run it. The same program text as the reference's main, against nsfsi_host.hpp.
//
//     nsfsi_main [ConfigFile] [output-folder]      (defaults: ./ConfigFile, ./output)
#include <iostream>
#include <string>

#include "nsfsi_host.hpp"

int main(int argc, char** argv) {
  const std::string configPath = argc > 1 ? argv[1] : "ConfigFile";
  const std::string outputDir = argc > 2 ? argv[2] : "output";
  nsfsi::ConfigSettings params(configPath);
  if (params.errorOccurred) return -1;
  try {
    nsfsi::Simulation simulation(params, 0, outputDir);
    simulation.run();
  } catch (const nsfsi::Error& e) {
    std::cerr << e.what() << std::endl;
    return 1;
  }
  return 0;
}
