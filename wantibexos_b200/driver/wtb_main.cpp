// wtb_bse: reads the deck from stdin (like `wtb.x < deck`) and runs the BSE path.
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <iterator>
#include <string>

#include "../../include/wtb_driver.h"

int main() {
  std::string deck((std::istreambuf_iterator<char>(std::cin)), std::istreambuf_iterator<char>());
  const char* dev = std::getenv("WTBG_DEVICE");
  char err[1024] = {0};
  if (wtb_run(deck.c_str(), dev ? std::atoi(dev) : 0, nullptr, err, sizeof err) != 0) {
    std::fprintf(stderr, "%s\n", err);
    return 1;
  }
  return 0;
}
