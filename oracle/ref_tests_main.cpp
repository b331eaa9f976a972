// Runs the reference's own image tests (src/Ray/tests/test_mesh_lights.cpp,
// test_texture.cpp), compiled unchanged, against this library: their
// Ray::CreateRenderer calls resolve to include/raygpu_factory.cpp, which
// returns the GPU renderer for every backend flag they loop over. The tests
// exit(-1) on a failed check (test_common.h); reaching the end prints OK.
#include <cstdio>

void test_mesh_lights();
void test_texture();

int main() {
    test_mesh_lights();
    test_texture();
    puts("OK");
    return 0;
}
