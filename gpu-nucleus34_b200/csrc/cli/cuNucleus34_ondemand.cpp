// Drop-in for the reference's on-demand program (nucleus/cuNucleus34_ondemand.cu:308-784):
//   cuNucleus34_ondemand <dataset file> [results output file]
// Memory is O(triangles): cliques are re-enumerated through the edge ->
// triangle incidence whenever the peel needs them.
#include "driver.h"

int main(int argc, char **argv)
{
	return rec::run_program({false, "b200-nucleus34-ondemand", "1.0.0"}, argc, argv);
}
