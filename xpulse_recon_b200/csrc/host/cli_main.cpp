// cli_main.cpp -- xprecon: drop-in for the reference's XPRecon command line
// (src/main.cpp:62-136): `xprecon -template | <json_file> | <json>`.
// Exit codes: 0 ok, -1 bad arguments, -2 bad parameters, -3 reconstruction error.
#include <cstdio>
#include <cstring>
#include <iostream>
#include <string>

#include "../../../include/xpr.h"

static void usage()
{
    std::cout << "xprecon -template|<json_file>|<json>" << std::endl;
    std::cout << "\t-template : Output in stdout a default JSON file" << std::endl;
    std::cout << "\t<json_file> : path to the parameters file" << std::endl;
    std::cout << "\t<json> : parameters as a JSON string (starting with a '{')" << std::endl;
}

int main(int argc, char *argv[])
{
    if (argc < 2) {
        usage();
        return -1;
    }
    if (std::string(argv[1]) == "-template") {
        std::string buf((size_t)xpr_template_json(nullptr, 0) + 1, '\0');
        xpr_template_json(&buf[0], buf.size());
        std::cout << buf.c_str() << std::endl;
        return 0;
    }
    return xpr_run(argv[1]);
}
