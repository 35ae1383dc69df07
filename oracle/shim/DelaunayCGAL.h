// TEST INFRASTRUCTURE ONLY -- stand-in for the reference's CGAL boundary header
// (inc/models/DelaunayCGAL.h of abaso/cellGPU), used to compile the reference's own CPU sources
// into oracle/_ref without CGAL (not installed here). It declares the same names the reference
// uses -- Point, LPoint, Iso_rectangle, PDT (periodic 2D Delaunay triangulation with face/vertex
// iterators and circulators) and the DelaunayCGAL class -- and implements them with the oracle's
// exact-predicate Delaunay code (cg_oracle.c). For points in general position the Delaunay
// triangulation is unique, so these answer what CGAL would.
//
// Conventions of this stand-in (CGAL leaves them unspecified): faces are enumerated with the
// smallest cell index first, in cell order then counter-clockwise slot order; vertex rows and
// circulators start at the smallest neighbour index; a face's vertex(i) are (c, a, b)
// counter-clockwise and neighbor(i) is the face opposite vertex(i); dual() is the circumcentre
// wrapped into the box.
#ifndef DELAUNAYCGAL_H
#define DELAUNAYCGAL_H

#include <map>
#include <utility>
#include <vector>

#include "std_include.h"
#include "vector_types.h"
#include "../cg_oracle.h"

using namespace std;

class Point {
  public:
    Point() : x_(0), y_(0) {}
    Point(double x, double y) : x_(x), y_(y) {}
    double x() const { return x_; }
    double y() const { return y_; }

  private:
    double x_, y_;
};
typedef Point LPoint;

class Iso_rectangle {
  public:
    Iso_rectangle(double x0, double y0, double x1, double y1) : x0_(x0), y0_(y0), x1_(x1), y1_(y1) {}
    double xmin() const { return x0_; }
    double ymin() const { return y0_; }
    double xmax() const { return x1_; }
    double ymax() const { return y1_; }

  private:
    double x0_, y0_, x1_, y1_;
};

class PDT {
  public:
    typedef ::Point Point;
    struct Vertex {
        int info_;
        int &info() { return info_; }
    };
    struct Face;
    typedef Face *Face_handle;
    struct Face {
        PDT *owner;
        int v[3];   // cell indices, counter-clockwise
        int nb[3];  // face opposite v[i]
        Vertex *vertex(int i) { return &owner->verts[v[i]]; }
        Face_handle neighbor(int i) { return &owner->faces[nb[i]]; }
    };
    typedef Vertex *Vertex_handle;

    class Face_iterator {
      public:
        Face_iterator(Face *p) : p_(p) {}
        Face_iterator &operator++() { ++p_; return *this; }
        bool operator!=(const Face_iterator &o) const { return p_ != o.p_; }
        Face *operator->() const { return p_; }
        operator Face_handle() const { return p_; }

      private:
        Face *p_;
    };
    class Vertex_iterator {
      public:
        Vertex_iterator(PDT *t, int i) : t_(t), i_(i) {}
        Vertex_iterator &operator++() { ++i_; return *this; }
        bool operator!=(const Vertex_iterator &o) const { return i_ != o.i_; }
        Vertex *operator->() const { return &t_->verts[i_]; }
        PDT *t_;
        int i_;
    };
    // neighbours of a vertex, counter-clockwise
    class Vertex_circulator {
      public:
        Vertex_circulator(const Vertex_iterator &v) : t_(v.t_), c_(v.i_), k_(0) {}
        Vertex_circulator &operator++() { k_ = (k_ + 1) % t_->nn[c_]; return *this; }
        Vertex *operator->() const { return &t_->verts[t_->nbr[(size_t)c_ * t_->K + k_]]; }

      private:
        PDT *t_;
        int c_, k_;
    };
    // faces around a vertex, counter-clockwise, starting at (c, nbr[0], nbr[1])
    class Face_circulator {
      public:
        Face_circulator(const Vertex_iterator &v) : t_(v.t_), c_(v.i_), k_(0) {}
        Face_circulator &operator++() { k_ = (k_ + 1) % t_->nn[c_]; return *this; }
        operator Face_handle() const { return &t_->faces[t_->tri[(size_t)c_ * t_->K + k_]]; }

      private:
        PDT *t_;
        int c_, k_;
    };

    template <class It>
    PDT(It first, It last, const Iso_rectangle &dom)
    {
        std::vector<std::pair<Point, int> > pts(first, last);
        int n = (int)pts.size();
        box[0] = dom.xmax() - dom.xmin();
        box[1] = dom.ymax() - dom.ymin();
        K = 32;
        pos.assign(2 * (size_t)n, 0.0);
        for (int i = 0; i < n; ++i) {
            pos[2 * (size_t)pts[i].second] = pts[i].first.x();
            pos[2 * (size_t)pts[i].second + 1] = pts[i].first.y();
        }
        nn.assign(n, 0);
        nbr.assign((size_t)n * K, -1);
        if (cgo_periodic_delaunay(n, pos.data(), box, K, nn.data(), nbr.data()) != 0)
            throw std::runtime_error("stand-in periodic Delaunay failed");
        verts.resize(n);
        for (int i = 0; i < n; ++i) verts[i].info_ = i;
        // faces: owner = smallest index
        tri.assign((size_t)n * K, -1);
        for (int c = 0; c < n; ++c)
            for (int k = 0; k < nn[c]; ++k) {
                int a = nbr[(size_t)c * K + k], b = nbr[(size_t)c * K + (k + 1) % nn[c]];
                if (c < a && c < b) {
                    Face f;
                    f.owner = this;
                    f.v[0] = c;
                    f.v[1] = a;
                    f.v[2] = b;
                    tri[(size_t)c * K + k] = (int)faces.size();
                    faces.push_back(f);
                }
            }
        for (int c = 0; c < n; ++c)
            for (int k = 0; k < nn[c]; ++k) {
                if (tri[(size_t)c * K + k] >= 0) continue;
                int a = nbr[(size_t)c * K + k], b = nbr[(size_t)c * K + (k + 1) % nn[c]];
                int o = a < b ? a : b, nxt = (o == a) ? b : c;
                tri[(size_t)c * K + k] = tri[(size_t)o * K + slot(o, nxt)];
            }
        for (size_t f = 0; f < faces.size(); ++f)
            for (int i = 0; i < 3; ++i) {
                int q = faces[f].v[(i + 1) % 3], r = faces[f].v[(i + 2) % 3];
                int s = slot(q, r);
                faces[f].nb[i] = tri[(size_t)q * K + (s + nn[q] - 1) % nn[q]];
            }
        for (size_t f = 0; f < faces.size(); ++f) faces[f].owner = this;
    }
    void convert_to_1_sheeted_covering() {}
    Face_iterator faces_begin() { return Face_iterator(faces.data()); }
    Face_iterator faces_end() { return Face_iterator(faces.data() + faces.size()); }
    Vertex_iterator vertices_begin() { return Vertex_iterator(this, 0); }
    Vertex_iterator vertices_end() { return Vertex_iterator(this, (int)verts.size()); }
    Point dual(Face_handle f)
    {
        double ra[2], rb[2], q[2];
        int c = f->v[0], a = f->v[1], b = f->v[2];
        cgo_min_dist(box, &pos[2 * (size_t)a], &pos[2 * (size_t)c], ra);
        cgo_min_dist(box, &pos[2 * (size_t)b], &pos[2 * (size_t)c], rb);
        double an = ra[0] * ra[0] + ra[1] * ra[1], bn = rb[0] * rb[0] + rb[1] * rb[1];
        double den = 0.5 / (ra[0] * rb[1] - ra[1] * rb[0]);
        q[0] = pos[2 * (size_t)c] + den * (an * rb[1] - ra[1] * bn);
        q[1] = pos[2 * (size_t)c + 1] + den * (ra[0] * bn - an * rb[0]);
        cgo_put_in_box(box, q);
        return Point(q[0], q[1]);
    }

    std::vector<Vertex> verts;
    std::vector<Face> faces;
    std::vector<int> nn, nbr, tri;
    std::vector<double> pos;
    double box[2];
    int K;

  private:
    int slot(int c, int v) const
    {
        for (int k = 0; k < nn[c]; ++k)
            if (nbr[(size_t)c * K + k] == v) return k;
        throw std::runtime_error("stand-in: inconsistent triangulation");
    }
};

typedef PDT::Vertex_handle Vertex_handle;
typedef PDT::Face_handle Face_handle;
typedef PDT::Vertex_circulator Vertex_circulator;

class DelaunayCGAL {
  public:
    vector<vector<int> > allneighs;

    void PeriodicTriangulation(vector<pair<Point, int> > &V, Dscalar bxx, Dscalar bxy, Dscalar byx, Dscalar byy)
    {
        (void)bxy;
        (void)byx;
        PeriodicTriangulationSquareDomain(V, bxx, byy);
    }
    void PeriodicTriangulationNineSheeted(vector<pair<Point, int> > &V, Dscalar bxx, Dscalar bxy, Dscalar byx,
                                          Dscalar byy)
    {
        PeriodicTriangulation(V, bxx, bxy, byx, byy);
    }
    void PeriodicTriangulationSquareDomain(vector<pair<Point, int> > &V, Dscalar boxX, Dscalar boxY)
    {
        int n = (int)V.size();
        const int K = 32;
        vector<double> pos(2 * (size_t)n);
        for (int i = 0; i < n; ++i) {
            pos[2 * (size_t)V[i].second] = V[i].first.x();
            pos[2 * (size_t)V[i].second + 1] = V[i].first.y();
        }
        vector<int> nn(n), nbr((size_t)n * K);
        double box[2] = {boxX, boxY};
        allneighs.assign(n, vector<int>());
        if (cgo_periodic_delaunay(n, pos.data(), box, K, nn.data(), nbr.data()) != 0) return;
        for (int i = 0; i < n; ++i) allneighs[i].assign(&nbr[(size_t)i * K], &nbr[(size_t)i * K] + nn[i]);
    }
    // neighbours of V[0] (at the origin of the relative coordinates the reference passes),
    // counter-clockwise, as indices into V (the reference stores those in the vertex info)
    bool LocalTriangulation(const vector<pair<LPoint, int> > &V, vector<int> &neighs)
    {
        neighs.clear();
        int m = (int)V.size() - 1;
        if (m < 3) return false;
        vector<double> rel(2 * (size_t)m);
        for (int i = 0; i < m; ++i) {
            rel[2 * (size_t)i] = V[i + 1].first.x() - V[0].first.x();
            rel[2 * (size_t)i + 1] = V[i + 1].first.y() - V[0].first.y();
        }
        vector<int> out(m + 1);
        int z = cgo_local_star(m, rel.data(), m + 1, out.data());
        if (z <= 0) return false;
        for (int k = 0; k < z; ++k) neighs.push_back(V[out[k] + 1].second);
        return true;
    }
};

#endif
