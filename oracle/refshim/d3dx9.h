/*
 * Oracle test infrastructure: headless stand-ins for the Direct3D 9 types that
 * the reference's headers declare.  There is no rendering: a vertex buffer is a
 * plain host allocation so that code paths which fill one still compile.
 */
#ifndef LENIA_REFSHIM_D3DX9_H
#define LENIA_REFSHIM_D3DX9_H

#include <stdint.h>
#include <stdlib.h>

typedef uint32_t D3DCOLOR;

#define D3DCOLOR_XRGB(r, g, b) \
    ((D3DCOLOR)((0xffu << 24) | (((r) & 0xff) << 16) | (((g) & 0xff) << 8) | ((b) & 0xff)))

#define D3DFVF_XYZ 0x002
#define D3DFVF_NORMAL 0x010
#define D3DFVF_DIFFUSE 0x040
#define D3DLOCK_DISCARD 0x2000

typedef int D3DDEVTYPE;

struct D3DXCOLOR {
    float r, g, b, a;
    D3DXCOLOR() : r(0), g(0), b(0), a(0) {}
    D3DXCOLOR(float r_, float g_, float b_, float a_) : r(r_), g(g_), b(b_), a(a_) {}
    D3DXCOLOR(D3DCOLOR c)
        : r(((c >> 16) & 0xff) / 255.0f), g(((c >> 8) & 0xff) / 255.0f),
          b((c & 0xff) / 255.0f), a(((c >> 24) & 0xff) / 255.0f) {}
    operator D3DCOLOR() const
    {
        return ((D3DCOLOR)(a * 255.0f) << 24) | ((D3DCOLOR)(r * 255.0f) << 16) |
               ((D3DCOLOR)(g * 255.0f) << 8) | (D3DCOLOR)(b * 255.0f);
    }
};

struct D3DXVECTOR3 { float x, y, z; };
struct D3DXVECTOR4 { float x, y, z, w; };
struct D3DXMATRIX { float m[4][4]; };
struct D3DLIGHT9 { int Type; };

struct IDirect3DDevice9 { int dummy; };

/* A lockable buffer backed by host memory, sized on first lock. */
struct IDirect3DVertexBuffer9 {
    void *mem;
    size_t bytes;
    long Lock(unsigned, unsigned, void **p, unsigned)
    {
        *p = mem;
        return 0;
    }
    long Unlock() { return 0; }
};

struct IDirect3DIndexBuffer9 {
    void *mem;
    size_t bytes;
    long Lock(unsigned, unsigned, void **p, unsigned)
    {
        *p = mem;
        return 0;
    }
    long Unlock() { return 0; }
};

#endif
