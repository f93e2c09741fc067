// Command-line program with the reference's interface (main.cu:9-93):
//   ftsp_main -p param [-i id] [-s dir] [--omega f] [--psi f] [--seq f]
//             [--screenprint] [--fp32|--fp64] [--si|--pc] [--seed N] [--device N]
#include "ftsp_host.h"

int main(int argc, char** argv) { return ftsp_main(argc, argv); }
