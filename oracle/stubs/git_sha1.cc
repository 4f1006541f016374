// Version strings for the reference's --version flag (hybrid_bfs_main.cc:119-121).
// Its build system generates this file from git_sha1.cc.in; the oracle build
// has no git checkout of the reference, so the tag is fixed.
#include "git_sha1.h"
const char g_GIT_SHA1[] = "unknown";
const char g_GIT_TAG[] = "reference-serial-elision";
