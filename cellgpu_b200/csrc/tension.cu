// cellgpu_b200 -- line tension of the Voronoi model (VoronoiQuadraticEnergyWithTension,
// src/models/voronoiQuadraticEnergyWithTension.cpp) and of the vertex model
// (VertexQuadraticEnergyWithTension, src/models/vertexQuadraticEnergyWithTension.cpp). Included by
// system.cu.
//
// Cells carry an integer type (Simple2DCell::setCellType, src/models/Simple2DCell.cpp:219-230).
// With tension on, every Voronoi edge between cells of different types carries gamma (one value,
// setSurfaceTension(g)) or gamma[type_self * ntypes + type_other] (setSurfaceTension(vector), a
// symmetric matrix) per unit length. The forces are those of the reference: at every Voronoi
// vertex each of its three cells contributes the derivative of its own unlike edges, i.e. the
// gradient of sum_cells [KA (A-A0)^2 + KP (P-P0)^2 + sum over the cell's unlike edges of
// gamma l] -- in the scatter form here each cell simply adds its unlike-edge term to its energy.
// The energy, as the reference's computeEnergy (:101-159), counts each unlike edge once.
//
// Vertex model: each force set (vertex, cell) also carries -gamma times the unit vector from the
// cell's next vertex to the vertex when the cell across that edge has another type, so every edge
// contributes its gradient once to each of its two vertices: the forces are minus the gradient of
// the quadratic energy plus gamma l over every unlike edge once, and that is the energy reported
// (the reference leaves this model's computeEnergy unimplemented).

static void drop_graphs(cg_system *s)
{
    cudaStreamSynchronize(s->stream);
    for (auto &g : s->graphs) release_graph(g);  // graphs captured the old arguments
    s->graphs.clear();
}

static int tension_alloc(cg_system *s)
{
    if (!s->ctype) {
        CG_TRY(dalloc(s, &s->ctype, s->N));  // zeroed: every cell of type 0
        CG_TRY(dalloc(s, &s->TE, s->N));
    }
    return CG_OK;
}

extern "C" int cg_set_cell_types(cg_system *s, const int *types)
{
    if (!s || !types) return set_err(CG_ERR_ARG, "bad args");
    for (int i = 0; i < s->N; ++i)
        if (types[i] < 0) return set_err(CG_ERR_ARG, "cell types must be >= 0");
    if (s->tension_mode == 2)
        for (int i = 0; i < s->N; ++i)
            if (types[i] >= s->ntypes) return set_err(CG_ERR_ARG, "cell type outside the tension matrix");
    CG_TRY(tension_alloc(s));
    return h2d(s, s->ctype, types, sizeof(int) * s->N);
}

extern "C" int cg_set_tension(cg_system *s, double gamma)
{
    if (!s || !(gamma == gamma)) return set_err(CG_ERR_ARG, "bad args");
    CG_TRY(tension_alloc(s));
    s->gamma = gamma;
    s->tension_mode = gamma != 0.0 ? 1 : 0;
    drop_graphs(s);
    return CG_OK;
}

extern "C" int cg_set_tension_matrix(cg_system *s, int ntypes, const double *gamma)
{
    if (!s || ntypes < 0 || (ntypes > 0 && !gamma))
        return set_err(CG_ERR_ARG, "bad args");
    // The reference weighs each edge by the matrix entry of one fixed ordering of its two cells'
    // types, and its computeEnergy by another; the two agree (and the forces are the gradient of
    // an energy) only for a symmetric matrix, which is what setSurfaceTension documents.
    for (int a = 0; a < ntypes; ++a)
        for (int b = 0; b < a; ++b)
            if (gamma[a * ntypes + b] != gamma[b * ntypes + a])
                return set_err(CG_ERR_ARG, "the tension matrix must be symmetric");
    CG_TRY(tension_alloc(s));
    if (ntypes == 0) {
        s->tension_mode = 0;
        drop_graphs(s);
        return CG_OK;
    }
    std::vector<int> types(s->N);
    CG_TRY(d2h(s, types.data(), s->ctype, sizeof(int) * s->N));
    for (int t : types)
        if (t >= ntypes) return set_err(CG_ERR_ARG, "cell type outside the tension matrix");
    if (s->tmat && s->ntypes < ntypes) s->tmat = nullptr;  // (the old block stays in the arena)
    if (!s->tmat) CG_TRY(dalloc(s, &s->tmat, (size_t)ntypes * ntypes));
    CG_TRY(h2d(s, s->tmat, gamma, sizeof(double) * (size_t)ntypes * ntypes));
    s->ntypes = ntypes;
    s->tension_mode = 2;
    drop_graphs(s);
    return CG_OK;
}
