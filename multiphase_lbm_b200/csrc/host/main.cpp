// main.cpp -- the `mlbm` program: a drop-in for the reference's
// `multiphaselbm <commandFile>` (src/main.cc:4-17): read the command file,
// open Stats.txt, run the time loop on the GPU.
#include <cstdio>
#include <iostream>

#include "../../../include/mlbm_driver.h"

int main(int argc, char const* argv[]) {
  if (argc != 2) {
    std::cout << "Usage: " << argv[0] << " commandFile" << std::endl;
    return 0;
  }
  mlbm_driver* box = nullptr;
  if (mlbm_driver_create(&box)) {
    std::cerr << mlbm_last_error() << std::endl;
    return 1;
  }
  std::cout << "Opening file : " << argv[1] << std::endl;
  int rc = 0;
  mlbm_status st = mlbm_driver_read(box, argv[1]);
  if (!st) st = mlbm_driver_init(box);
  int64_t step0 = 0, step_max = 0;
  mlbm_driver_info(box, &step0, &step_max, nullptr, nullptr, nullptr, nullptr,
                   nullptr);
  if (!st) st = mlbm_driver_run(box, 0);
  if (st) {
    std::cerr << "mlbm: " << mlbm_status_string(st) << ": " << mlbm_last_error()
              << std::endl;
    rc = 1;
  }
  mlbm_driver_destroy(box);
  return rc;
}
