// Reader for the reference's scene-file grammar (scene/scene_file.hpp:62-131) and
// its Wavefront OBJ subset (geometry/obj.hpp:45-70), building a HostScene with the
// same object, light and material order as the reference's readScene.
#pragma once

#include "host_scene.hpp"

#include <filesystem>
#include <stdexcept>
#include <string>

namespace albedo_b200 {

// What readScene throws for input it cannot accept; the message names the line
// as the reference's SceneParseError does (scene/scene_file.cpp:1051-1056).
class SceneParseError : public std::runtime_error {
public:
    SceneParseError(std::size_t line, const std::string& problem);
    std::size_t line() const noexcept { return line_number; }

private:
    std::size_t line_number;
};

// Reads the scene file at `path`; meshes are found beside it. Throws
// SceneParseError, or std::runtime_error naming the path if it cannot be opened.
HostScene readSceneFile(const std::filesystem::path& path);

// Reads scene text; `base_directory` empty means meshes are refused.
HostScene readSceneText(const std::string& text, const std::filesystem::path& base_directory);

} // namespace albedo_b200
