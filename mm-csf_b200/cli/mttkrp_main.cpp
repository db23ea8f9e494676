// placeholder CLI (filled in with the reference's flags)
#include <cstdio>
#include "mmcsf.h"
int main() { printf("mmcsf %d\n", mmcsf_version()); return 0; }
