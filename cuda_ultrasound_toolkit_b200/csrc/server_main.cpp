// cutb_transfer_server: serves beamform / motion-detection / image-correlation requests of
// libcuda_transfer.so clients (upstream test_app/src/main.cpp + TestApp::run).
//
//   cutb_transfer_server [--name NAME] [--data-bytes N] [--max-commands K] [--timeout-ms T]
//
// Prints "ready <name>" on stdout once the socket and the shared memory exist. Exits 0 after K
// commands (0 = no limit) or T ms without a command (default one hour, as upstream).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/cuda_toolkit_b200_server.h"

int main(int argc, char** argv)
{
    const char* name = nullptr;
    unsigned long long bytes = 0;
    int max_commands = 0, timeout_ms = 60 * 60 * 1000;
    for (int i = 1; i + 1 < argc; i += 2) {
        if (!strcmp(argv[i], "--name"))
            name = argv[i + 1];
        else if (!strcmp(argv[i], "--data-bytes"))
            bytes = strtoull(argv[i + 1], nullptr, 0);
        else if (!strcmp(argv[i], "--max-commands"))
            max_commands = atoi(argv[i + 1]);
        else if (!strcmp(argv[i], "--timeout-ms"))
            timeout_ms = atoi(argv[i + 1]);
        else {
            fprintf(stderr, "unknown option %s\n", argv[i]);
            return 2;
        }
    }
    cutb_server* s = cutb_server_create(name, bytes);
    if (!s) return 1;
    printf("ready %s\n", name ? name : "(default)");
    fflush(stdout);
    const int handled = cutb_server_serve(s, max_commands, timeout_ms);
    cutb_server_destroy(s);
    return handled < 0 ? 1 : 0;
}
