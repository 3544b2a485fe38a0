// gsjd executable: the daemon lives in libgsjd.so (gsjd_main).
#include "../../../include/gsjd.h"

int main(int argc, char** argv) { return gsjd_main(argc, argv); }
