/* Declarations of the Lua 5.4 C API names that the reference's structure
 * sources mention. Test infrastructure for the oracle build only: Lua is
 * absent here, and the oracle never runs a structure script, so every
 * definition (refshim/structstubs.cpp) aborts when called. */
#pragma once
extern "C" {
struct lua_State;
typedef int (*lua_CFunction)(lua_State *);
typedef double lua_Number;
typedef long long lua_Integer;
#define LUA_OK 0
#define LUA_ERRSYNTAX 3
#define LUA_ERRFILE 6
#define LUA_TNIL 0
#define LUA_TBOOLEAN 1
#define LUA_TLIGHTUSERDATA 2
#define LUA_TNUMBER 3
#define LUA_TSTRING 4
#define LUA_TTABLE 5
#define LUA_TFUNCTION 6
#define LUA_TUSERDATA 7
#define LUA_MULTRET (-1)
lua_State *luaL_newstate(void);
void luaL_openlibs(lua_State *L);
int luaL_loadstring(lua_State *L, const char *s);
int luaL_getmetatable(lua_State *L, const char *n);
void lua_close(lua_State *L);
int lua_type(lua_State *L, int i);
lua_Number lua_tonumber(lua_State *L, int i);
lua_Integer lua_tointeger(lua_State *L, int i);
const char *lua_tostring(lua_State *L, int i);
void lua_pushnumber(lua_State *L, lua_Number n);
void lua_pushinteger(lua_State *L, lua_Integer n);
void lua_pushstring(lua_State *L, const char *s);
void lua_pushvalue(lua_State *L, int i);
void lua_pushlightuserdata(lua_State *L, void *p);
int lua_getglobal(lua_State *L, const char *n);
void lua_setglobal(lua_State *L, const char *n);
int lua_setmetatable(lua_State *L, int i);
void *lua_newuserdata(lua_State *L, unsigned long sz);
void *lua_touserdata(lua_State *L, int i);
void lua_pop(lua_State *L, int n);
int lua_pcall(lua_State *L, int a, int r, int e);
void lua_call(lua_State *L, int a, int r);
int lua_isnil(lua_State *L, int i);
int lua_gettop(lua_State *L);
void lua_register(lua_State *L, const char *n, lua_CFunction f);
int lua_isnumber(lua_State *L, int i);
int lua_isstring(lua_State *L, int i);
void lua_createtable(lua_State *L, int a, int b);
void lua_settable(lua_State *L, int i);
void lua_pushcfunction(lua_State *L, lua_CFunction f);
void lua_setfield(lua_State *L, int i, const char *k);
int lua_getfield(lua_State *L, int i, const char *k);
int luaL_newmetatable(lua_State *L, const char *n);
void lua_pushboolean(lua_State *L, int b);
int lua_toboolean(lua_State *L, int i);
void lua_settop(lua_State *L, int i);
int lua_rawgeti(lua_State *L, int i, lua_Integer n);
int lua_geti(lua_State *L, int i, lua_Integer n);
void lua_seti(lua_State *L, int i, lua_Integer n);
int lua_next(lua_State *L, int i);
void lua_pushnil(lua_State *L);
int luaL_dofile(lua_State *L, const char *f);
int luaL_loadfile(lua_State *L, const char *f);
void *luaL_checkudata(lua_State *L, int i, const char *n);
int lua_isuserdata(lua_State *L, int i);
int lua_istable(lua_State *L, int i);
int lua_isfunction(lua_State *L, int i);
int lua_isinteger(lua_State *L, int i);
unsigned long long lua_rawlen(lua_State *L, int i);
}
