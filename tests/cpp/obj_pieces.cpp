// The OBJ reader gives the same mesh, or the same error, however many pieces
// (threads) it splits a file into. Compiled together with the reader's source;
// for each OBJ file named on the command line (and budgets: vertices, texture
// coordinates, triangles) it reads the file in 1, 2, 3, 5, 8 and 13 pieces and
// prints one line: "same" or "differs", the outcome ("ok" with counts, or the
// error message).
#include "host/scene_file.cpp"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>

using namespace albedo_b200;

namespace {

std::string outcome(std::string_view text, const ObjBudget& budget, unsigned pieces)
{
    try {
        const ObjMesh mesh{parseObj(text, budget, pieces)};
        std::string out{std::format("ok {} {} {} {} ", mesh.positions.size(), mesh.uvs.size(), mesh.faces.size(),
                                    mesh.texture_faces.size())};
        std::uint64_t h{1469598103934665603ull};
        const auto mix = [&](const void* data, std::size_t bytes) {
            const auto* b = static_cast<const unsigned char*>(data);
            for (std::size_t i{0}; i < bytes; ++i) {
                h = (h ^ b[i]) * 1099511628211ull;
            }
        };
        mix(mesh.positions.data(), mesh.positions.size() * sizeof(Vec3));
        mix(mesh.uvs.data(), mesh.uvs.size() * sizeof(mesh.uvs[0]));
        mix(mesh.faces.data(), mesh.faces.size() * sizeof(mesh.faces[0]));
        mix(mesh.texture_faces.data(), mesh.texture_faces.size() * sizeof(mesh.texture_faces[0]));
        return out + std::format("{:016x}", h);
    } catch (const ObjError& error) {
        return std::string{"error "} + error.what();
    }
}

} // namespace

int main(int argc, char** argv)
{
    for (int i{1}; i + 3 < argc; i += 4) {
        std::ifstream file{argv[i], std::ios::binary};
        const std::string text{std::istreambuf_iterator<char>{file}, std::istreambuf_iterator<char>{}};
        const ObjBudget budget{.vertices = std::stoull(argv[i + 1]), .texture_coordinates = std::stoull(argv[i + 2]),
                               .triangles = std::stoull(argv[i + 3])};
        const std::string one{outcome(text, budget, 1)};
        bool same{true};
        for (const unsigned pieces : {2u, 3u, 5u, 8u, 13u}) {
            same = same && outcome(text, budget, pieces) == one;
        }
        std::printf("%s\t%s\n", same ? "same" : "differs", one.c_str());
    }
    return 0;
}
