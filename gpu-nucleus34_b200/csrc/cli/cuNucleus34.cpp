// Drop-in for the reference's direct program (nucleus/cuNucleus34.cu:144-839):
//   cuNucleus34 <dataset file> [parts] [results output file]
// Four-cliques and the triangle -> clique incidence are materialised on the
// device; the k file pairs each canonical triangle with its own k.
#include "driver.h"

int main(int argc, char **argv)
{
	return rec::run_program({true, "b200-nucleus34-direct", "1.0.0"}, argc, argv);
}
