// main.cu -- drop-in CLI with the reference's contract (main.cu:4-43):
//   <init load value> <load type x> <load type y> <load type xy> <time steps> <load value>
// Exit status 0 on success, 1 on an exception (message on stderr), -1 (255) on a CUDA
// error.  The reference always reads the sixth value (main.cu:17-18), so five values
// fail there with an exception; here they fail with the usage message, also status 1.
#include <string>

#include "EffPlast2D.h"

int main(int argc, char** argv) {
  try {
    const std::string err_info = "ERROR:  missing arguments\n USAGE: " + std::string(argv[0]) +
                                 " <init load value> <init load type>.x <init load type>.y <init load type>.xy "
                                 "<time steps> [<load value>]";
    if (argc < 7) throw std::invalid_argument(err_info);

    const double init_load_value = std::stod(argv[1]);
    const std::array<double, 3> load_type = {std::stod(argv[2]), std::stod(argv[3]), std::stod(argv[4])};
    const unsigned int time_steps = std::stod(argv[5]);
    const double load_value = std::stod(argv[6]);

    EffPlast2D eff_plast(time_steps);
    if (NL <= 3) {
      eff_plast.ComputeEffModuli(init_load_value, load_type, load_value);
    } else {
      eff_plast.ComputeEffDamping(init_load_value, load_type, load_value);
    }
    return 0;
  } catch (const std::exception& e) {
    std::cerr << e.what() << "\n";
    return 1;
  }
}
