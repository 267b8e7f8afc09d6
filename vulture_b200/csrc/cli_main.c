/* Entry point of the vulture-b200 executable: the reference's command line
 * (src/vulture.c:77-197) on the GPU engine. */
#include "vhost.h"

int main(int argc, char **argv) { return vhost_main(argc, argv); }
