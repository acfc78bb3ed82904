// uegccd_zcode -- the drop-in for the reference's ZCode executable.
//
//   uegccd_zcode [Input [Twists]]   (UEGCCD_SCHEME=diis selects the Pulay DIIS scheme)
//
// Reads the Input file (default ./Input), writes Output, fort.58 and fort.59 in the
// working directory.  Twists, when given, lists the twist angles of the twist
// average, three numbers per line.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "../../include/uegccd.h"
#include "../../include/uegccd_host.h"

int main(int argc, char **argv)
{
    const char *input = argc > 1 ? argv[1] : "Input";
    const char *twists = argc > 2 ? argv[2] : nullptr;
    const char *sch = std::getenv("UEGCCD_SCHEME");
    const int scheme = (sch && std::string(sch) == "diis") ? UEGCCD_DIIS : UEGCCD_REPLAY;
    const int rc = uegccd_zcode(input, twists, scheme);
    if (rc < 0) {
        std::fprintf(stderr, "uegccd_zcode: %s\n", uegccd_zcode_last_error());
        return 1;
    }
    return 0;
}
