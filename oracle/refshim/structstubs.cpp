/* Link stubs for the oracle build of the reference's structure sources
 * (structure.cpp, structure_primitives.cpp).
 *
 * Test infrastructure only. Lua is absent here: the oracle builds Structure
 * objects directly and never runs a structure script, so the Lua C API, the
 * Lua-side structure functions (LuaUI::*) and the .ageom converter are never
 * reached; each aborts so that a stray call cannot pass silently. The Bitmap
 * preview used by Structure::print is a no-op. */
#include <bitmap3.h>
#include <lua_base.h>
#include <lua_structure.h>

#include <cstdio>
#include <cstdlib>

[[noreturn]] static void aeoracle_no_lua(const char *what) {
    std::fprintf(stderr, "aeoracle: Lua entry point called in the oracle build: %s\n", what);
    std::abort();
}

void Bitmap::G2BW(Grid2<double> &, std::string) {}

extern "C" {
lua_State *luaL_newstate(void) { aeoracle_no_lua("luaL_newstate"); }
void luaL_openlibs(lua_State *) { aeoracle_no_lua("luaL_openlibs"); }
int luaL_loadstring(lua_State *, const char *) { aeoracle_no_lua("luaL_loadstring"); }
void lua_close(lua_State *) { aeoracle_no_lua("lua_close"); }
void lua_call(lua_State *, int, int) { aeoracle_no_lua("lua_call"); }
int lua_pcall(lua_State *, int, int, int) { aeoracle_no_lua("lua_pcall"); }
int lua_getglobal(lua_State *, const char *) { aeoracle_no_lua("lua_getglobal"); }
void lua_setglobal(lua_State *, const char *) { aeoracle_no_lua("lua_setglobal"); }
int lua_isnil(lua_State *, int) { aeoracle_no_lua("lua_isnil"); }
void lua_pop(lua_State *, int) { aeoracle_no_lua("lua_pop"); }
void lua_pushlightuserdata(lua_State *, void *) { aeoracle_no_lua("lua_pushlightuserdata"); }
void lua_pushnumber(lua_State *, lua_Number) { aeoracle_no_lua("lua_pushnumber"); }
void lua_pushvalue(lua_State *, int) { aeoracle_no_lua("lua_pushvalue"); }
void lua_register(lua_State *, const char *, lua_CFunction) { aeoracle_no_lua("lua_register"); }
lua_Integer lua_tointeger(lua_State *, int) { aeoracle_no_lua("lua_tointeger"); }
lua_Number lua_tonumber(lua_State *, int) { aeoracle_no_lua("lua_tonumber"); }
}

int nearest_integer(lua_State *) { aeoracle_no_lua("nearest_integer"); }
std::string ageom_to_lua(std::filesystem::path const &) { aeoracle_no_lua("ageom_to_lua"); }

namespace lua_tools {
int lua_adaptive_trapeze_integral(lua_State *) { aeoracle_no_lua("trapz"); }
}

namespace LuaUI {
#define AEORACLE_LUAUI(f) int f(lua_State *) { aeoracle_no_lua(#f); }
AEORACLE_LUAUI(random_packing)
AEORACLE_LUAUI(structure_add_block)
AEORACLE_LUAUI(structure_add_coating)
AEORACLE_LUAUI(structure_add_cone)
AEORACLE_LUAUI(structure_add_conf_coating)
AEORACLE_LUAUI(structure_add_cylinder)
AEORACLE_LUAUI(structure_add_ellipsoid)
AEORACLE_LUAUI(structure_add_layer)
AEORACLE_LUAUI(structure_add_lua_def)
AEORACLE_LUAUI(structure_add_mesh)
AEORACLE_LUAUI(structure_add_sin_layer)
AEORACLE_LUAUI(structure_add_sphere)
AEORACLE_LUAUI(structure_add_vect_block)
AEORACLE_LUAUI(structure_add_vect_tri)
AEORACLE_LUAUI(structure_declare_parameter)
AEORACLE_LUAUI(structure_default_material)
AEORACLE_LUAUI(structure_set_flip)
AEORACLE_LUAUI(structure_set_loop)
#undef AEORACLE_LUAUI
}  // namespace LuaUI
