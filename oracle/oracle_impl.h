/*
 * Scalar-generic body of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 * Included by oracle.c with ORC_SCALAR (float|double), ORC_SFX (f32|f64) and
 * ORC_EPSILON defined.  Every routine cites the reference lines it restates.
 */
#define ORC_CAT2(a, b) a##_##b
#define ORC_CAT(a, b) ORC_CAT2(a, b)
#define FN(name) ORC_CAT(name, ORC_SFX)
#define S ORC_SCALAR
#define NE ORC_CAT(orc_ne, ORC_SFX)

/* ===================================================================== COO -> CSR
 * sparse_ops_cpu.cpp:24-134.  Validation order and messages follow combineCoo. */
int FN(orc_coo_to_csr)(int64_t rows, int64_t cols, int64_t count, const int64_t* row_indices,
                       const int64_t* col_indices, const S* values, int64_t* row_offsets,
                       int64_t* out_columns, S* out_values, int64_t* out_nnz)
{
    if (rows < 0 || cols < 0)
    {
        return orc_fail(ORC_INVALID_ARGUMENT, "cooToCsr dimensions must be non-negative");
    }
    if (count < 0)
    {
        return orc_fail(ORC_INVALID_ARGUMENT,
                        "cooToCsr row, column, and value arrays must have equal lengths");
    }
    for (int64_t position = 0; position < count; ++position)
    {
        const int64_t row = row_indices[position];
        const int64_t col = col_indices[position];
        if (row < 0 || row >= rows || col < 0 || col >= cols)
        {
            return orc_fail(ORC_OUT_OF_RANGE,
                            "cooToCsr coordinate out of range at triplet %lld: (%lld, %lld) for "
                            "matrix %lldx%lld",
                            (long long)position, (long long)row, (long long)col, (long long)rows,
                            (long long)cols);
        }
    }
    int64_t* permutation = (int64_t*)malloc((size_t)(count > 0 ? count : 1) * sizeof(int64_t));
    if (!permutation)
    {
        return orc_fail(ORC_NO_MEMORY, "oracle: out of memory");
    }
    int status = orc_stable_sort_pairs(count, row_indices, col_indices, permutation);
    if (status != ORC_OK)
    {
        free(permutation);
        return status;
    }
    /* combine in sorted (stable) order: first value verbatim, then += */
    int64_t combined = 0;
    for (int64_t r = 0; r <= rows; ++r)
    {
        row_offsets[r] = 0;
    }
    int64_t last_row = -1, last_col = -1;
    for (int64_t k = 0; k < count; ++k)
    {
        const int64_t source = permutation[k];
        const int64_t row = row_indices[source];
        const int64_t col = col_indices[source];
        if (combined > 0 && last_row == row && last_col == col)
        {
            out_values[combined - 1] += values[source];
        }
        else
        {
            out_columns[combined] = col;
            out_values[combined] = values[source];
            ++row_offsets[row + 1];
            ++combined;
            last_row = row;
            last_col = col;
        }
    }
    for (int64_t r = 0; r < rows; ++r)
    {
        row_offsets[r + 1] += row_offsets[r];
    }
    *out_nnz = combined;
    free(permutation);
    return ORC_OK;
}

/* ===================================================================== CSR SpMV
 * sparse_ops_cpu.cpp:214-233. */
int FN(orc_csr_spmv)(int64_t rows, int64_t cols, const int64_t* row_offsets, const int64_t* columns,
                     const S* values, const S* x, S* y)
{
    (void)cols;
    if (x == y && x != NULL)
    {
        return orc_fail(ORC_INVALID_ARGUMENT, "spmv input and output data must not alias");
    }
    for (int64_t row = 0; row < rows; ++row)
    {
        S sum = (S)0;
        for (int64_t position = row_offsets[row]; position < row_offsets[row + 1]; ++position)
        {
            sum += values[position] * x[columns[position]];
        }
        y[row] = sum;
    }
    return ORC_OK;
}

/* spmm: sparse_ops_cpu.cpp:244-270; dense matrices column-major (leading dimension = rows),
 * column by column, each row summed from zero in storage order. */
int FN(orc_csr_spmm)(int64_t rows, int64_t cols, const int64_t* row_offsets, const int64_t* columns,
                     const S* values, int64_t k, const S* input, S* output)
{
    if (input == output && input != NULL)
    {
        return orc_fail(ORC_INVALID_ARGUMENT, "spmm input and output data must not alias");
    }
    for (int64_t col = 0; col < k; ++col)
    {
        const S* b_column = input + col * cols;
        S* out_column = output + col * rows;
        for (int64_t row = 0; row < rows; ++row)
        {
            S sum = (S)0;
            for (int64_t position = row_offsets[row]; position < row_offsets[row + 1]; ++position)
            {
                sum += values[position] * b_column[columns[position]];
            }
            out_column[row] = sum;
        }
    }
    return ORC_OK;
}

/* ===================================================================== CG / PCG
 * iterative_solver_cpu.cpp:15-284 (validateOptions, validateSystem, jacobiInverse, solve). */
static double FN(orc_dot64)(int64_t n, const double* a, const double* b)
{
    double result = 0.0;
    for (int64_t i = 0; i < n; ++i)
    {
        result += a[i] * b[i];
    }
    return result;
}

static void FN(orc_multiply64)(int64_t n, const int64_t* row_offsets, const int64_t* columns,
                               const S* values, const double* input, double* output)
{
    for (int64_t row = 0; row < n; ++row)
    {
        double sum = 0.0;
        for (int64_t position = row_offsets[row]; position < row_offsets[row + 1]; ++position)
        {
            sum += (double)values[position] * input[columns[position]];
        }
        output[row] = sum;
    }
}

int FN(orc_pcg)(int64_t n, const int64_t* row_offsets, const int64_t* columns, const S* values,
                const S* rhs, S* solution, const orc_solver_options* options, int preconditioned,
                orc_solver_report* report)
{
    memset(report, 0, sizeof(*report));
    if (options->max_iterations < 0)
    {
        return orc_fail(ORC_INVALID_ARGUMENT, "iterative solver maxIterations must be non-negative");
    }
    if (!isfinite(options->relative_tolerance) || options->relative_tolerance < 0.0 ||
        options->relative_tolerance > 1.0 || !isfinite(options->absolute_tolerance) ||
        options->absolute_tolerance < 0.0)
    {
        return orc_fail(ORC_INVALID_ARGUMENT,
                        "iterative solver relative tolerance must be in [0, 1] and absolute "
                        "tolerance must be finite and non-negative");
    }
    if (rhs == solution && rhs != NULL)
    {
        return orc_fail(ORC_INVALID_ARGUMENT, "iterative solver rhs and solution must not alias");
    }
    if (row_offsets[0] != 0)
    {
        return orc_fail(ORC_INVALID_ARGUMENT,
                        "iterative solver requires CSR row offsets to start at zero and end at nnz");
    }
    const int64_t nnz = row_offsets[n];
    for (int64_t row = 0; row < n; ++row)
    {
        if (row_offsets[row] < 0 || row_offsets[row + 1] < row_offsets[row] ||
            row_offsets[row + 1] > nnz)
        {
            return orc_fail(ORC_INVALID_ARGUMENT, "iterative solver invalid CSR row offsets at row %lld",
                            (long long)row);
        }
    }
    for (int64_t position = 0; position < nnz; ++position)
    {
        if (columns[position] < 0 || columns[position] >= n)
        {
            return orc_fail(ORC_INVALID_ARGUMENT,
                            "iterative solver CSR column index out of range at position %lld",
                            (long long)position);
        }
        if (!isfinite((double)values[position]))
        {
            return orc_fail(ORC_INVALID_ARGUMENT,
                            "iterative solver CSR value is not finite at position %lld",
                            (long long)position);
        }
    }
    for (int64_t row = 0; row < n; ++row)
    {
        if (!isfinite((double)rhs[row]) || !isfinite((double)solution[row]))
        {
            return orc_fail(ORC_INVALID_ARGUMENT,
                            "iterative solver rhs and solution must be finite at row %lld",
                            (long long)row);
        }
    }

    const size_t size = (size_t)(n > 0 ? n : 1);
    double* x = (double*)malloc(size * sizeof(double));
    double* residual = (double*)malloc(size * sizeof(double));
    double* direction = (double*)malloc(size * sizeof(double));
    double* transformed = (double*)malloc(size * sizeof(double));
    double* matrix_direction = (double*)malloc(size * sizeof(double));
    double* inverse_diagonal = (double*)malloc(size * sizeof(double));
    int status = ORC_OK;
    if (!x || !residual || !direction || !transformed || !matrix_direction || !inverse_diagonal)
    {
        status = orc_fail(ORC_NO_MEMORY, "oracle: out of memory");
        goto done;
    }
    for (int64_t i = 0; i < n; ++i)
    {
        x[i] = (double)solution[i];
    }
    FN(orc_multiply64)(n, row_offsets, columns, values, x, matrix_direction);
    for (int64_t i = 0; i < n; ++i)
    {
        residual[i] = (double)rhs[i] - matrix_direction[i];
    }
    const double initial_squared = FN(orc_dot64)(n, residual, residual);
    if (!isfinite(initial_squared) || initial_squared < 0.0)
    {
        status = orc_fail(ORC_RUNTIME_ERROR, "iterative solver initial residual is not finite");
        goto done;
    }
    report->initial_residual = sqrt(initial_squared);
    report->final_residual = report->initial_residual;
    const double tolerance = fmax(options->absolute_tolerance,
                                  options->relative_tolerance * report->initial_residual);
    if (report->final_residual <= tolerance)
    {
        report->converged = 1;
        goto done;
    }
    const int use_jacobi = preconditioned && options->use_jacobi;
    if (use_jacobi)
    {
        /* jacobiInverse, iterative_solver_cpu.cpp:127-160 */
        for (int64_t row = 0; row < n; ++row)
        {
            int found = 0;
            double diagonal = 0.0, row_scale = 0.0;
            for (int64_t position = row_offsets[row]; position < row_offsets[row + 1]; ++position)
            {
                const double value = (double)values[position];
                row_scale = fmax(row_scale, fabs(value));
                if (columns[position] == row)
                {
                    diagonal += value;
                    found = 1;
                }
            }
            const double threshold = ORC_EPSILON * row_scale * 16.0;
            if (!found || !isfinite(diagonal) || diagonal <= threshold || !isfinite(1.0 / diagonal))
            {
                status = orc_fail(ORC_RUNTIME_ERROR,
                                  "pcg Jacobi diagonal is missing, non-positive, or near zero at row %lld",
                                  (long long)row);
                goto done;
            }
            inverse_diagonal[row] = 1.0 / diagonal;
        }
    }
    for (int64_t i = 0; i < n; ++i)
    {
        transformed[i] = use_jacobi ? inverse_diagonal[i] * residual[i] : residual[i];
        direction[i] = transformed[i];
    }
    double rho = FN(orc_dot64)(n, residual, transformed);
    if (!isfinite(rho) || rho <= 0.0)
    {
        status = orc_fail(ORC_RUNTIME_ERROR,
                          "iterative solver breakdown: preconditioned residual is not positive");
        goto done;
    }
    for (int iteration = 0; iteration < options->max_iterations; ++iteration)
    {
        FN(orc_multiply64)(n, row_offsets, columns, values, direction, matrix_direction);
        const double denominator = FN(orc_dot64)(n, direction, matrix_direction);
        if (!isfinite(denominator) || denominator <= 0.0)
        {
            status = orc_fail(ORC_RUNTIME_ERROR, "iterative solver breakdown: matrix is not numerically SPD");
            goto done;
        }
        const double alpha = rho / denominator;
        if (!isfinite(alpha))
        {
            status = orc_fail(ORC_RUNTIME_ERROR, "iterative solver breakdown: step size is not finite");
            goto done;
        }
        for (int64_t i = 0; i < n; ++i)
        {
            x[i] += alpha * direction[i];
            residual[i] -= alpha * matrix_direction[i];
        }
        report->iterations = iteration + 1;
        const double residual_squared = FN(orc_dot64)(n, residual, residual);
        if (!isfinite(residual_squared) || residual_squared < 0.0)
        {
            status = orc_fail(ORC_RUNTIME_ERROR, "iterative solver residual is not finite");
            goto done;
        }
        report->final_residual = sqrt(residual_squared);
        if (report->final_residual <= tolerance)
        {
            report->converged = 1;
            break;
        }
        for (int64_t i = 0; i < n; ++i)
        {
            transformed[i] = use_jacobi ? inverse_diagonal[i] * residual[i] : residual[i];
        }
        const double next_rho = FN(orc_dot64)(n, residual, transformed);
        if (!isfinite(next_rho) || next_rho <= 0.0)
        {
            status = orc_fail(ORC_RUNTIME_ERROR, "iterative solver breakdown in direction update");
            goto done;
        }
        const double beta = next_rho / rho;
        if (!isfinite(beta))
        {
            status = orc_fail(ORC_RUNTIME_ERROR, "iterative solver breakdown: direction scale is not finite");
            goto done;
        }
        for (int64_t i = 0; i < n; ++i)
        {
            direction[i] = transformed[i] + beta * direction[i];
        }
        rho = next_rho;
    }
    for (int64_t i = 0; i < n; ++i)
    {
        solution[i] = (S)x[i];
    }
    if (!report->converged && options->require_convergence)
    {
        status = orc_fail(ORC_RUNTIME_ERROR,
                          "iterative solver did not converge in %d iterations; final residual=%g",
                          report->iterations, report->final_residual);
    }
done:
    free(x);
    free(residual);
    free(direction);
    free(transformed);
    free(matrix_direction);
    free(inverse_diagonal);
    return status;
}

/* ===================================================================== Huber
 * robust_loss.h:27-51. */
int FN(orc_huber)(S squared_norm, S delta, S* cost, S* weight)
{
    if (!isfinite(squared_norm) || squared_norm < (S)0)
    {
        return orc_fail(ORC_INVALID_ARGUMENT,
                        "evaluateHuberLoss: squared residual norm must be finite and non-negative");
    }
    if (!isfinite(delta) || delta < (S)0)
    {
        return orc_fail(ORC_INVALID_ARGUMENT, "evaluateHuberLoss: delta must be finite and non-negative");
    }
    if (delta == (S)0 || squared_norm <= delta * delta)
    {
        *cost = (S)0.5 * squared_norm;
        *weight = (S)1;
        return ORC_OK;
    }
    const S norm = (S)sqrt(squared_norm);
    *cost = delta * norm - (S)0.5 * delta * delta;
    *weight = delta / norm;
    return ORC_OK;
}

/* ===================================================================== normal equations
 * block_normal_equations.cpp.  Crosses live in creation order (the reference's
 * _crossBlocks vector); each eliminated block keeps its adjacency as a linked
 * list in insertion order (the reference's _eliminatedAdjacency). */
struct NE
{
    int64_t P, L, bp, bl;
    S* primary_diagonal;
    S* eliminated_diagonal;
    S* primary_gradient;
    S* eliminated_gradient;
    int64_t cross_count, cross_capacity;
    int64_t* cross_primary;
    int64_t* cross_eliminated;
    int64_t* cross_next;
    S* cross_values;
    int64_t* adjacency_head;
    int64_t* adjacency_tail;
    int64_t* adjacency_size;
    int64_t pc_count, pc_capacity;
    int64_t* pc_row;
    int64_t* pc_col;
    S* pc_values;
};

NE* FN(orc_ne_create)(int64_t primary_count, int64_t eliminated_count, int64_t primary_size,
                      int64_t eliminated_size)
{
    if (primary_count < 0 || eliminated_count < 0 || primary_size <= 0 || eliminated_size <= 0)
    {
        orc_fail(ORC_INVALID_ARGUMENT,
                 "BlockNormalEquations: block counts must be non-negative and block sizes positive");
        return NULL;
    }
    NE* ne = (NE*)calloc(1, sizeof(NE));
    if (!ne)
    {
        return NULL;
    }
    ne->P = primary_count;
    ne->L = eliminated_count;
    ne->bp = primary_size;
    ne->bl = eliminated_size;
    ne->primary_diagonal = (S*)calloc((size_t)(primary_count * primary_size * primary_size) + 1, sizeof(S));
    ne->eliminated_diagonal =
        (S*)calloc((size_t)(eliminated_count * eliminated_size * eliminated_size) + 1, sizeof(S));
    ne->primary_gradient = (S*)calloc((size_t)(primary_count * primary_size) + 1, sizeof(S));
    ne->eliminated_gradient = (S*)calloc((size_t)(eliminated_count * eliminated_size) + 1, sizeof(S));
    ne->adjacency_head = (int64_t*)malloc(((size_t)eliminated_count + 1) * sizeof(int64_t));
    ne->adjacency_tail = (int64_t*)malloc(((size_t)eliminated_count + 1) * sizeof(int64_t));
    ne->adjacency_size = (int64_t*)calloc((size_t)eliminated_count + 1, sizeof(int64_t));
    for (int64_t l = 0; l < eliminated_count; ++l)
    {
        ne->adjacency_head[l] = -1;
        ne->adjacency_tail[l] = -1;
    }
    return ne;
}

void FN(orc_ne_destroy)(NE* ne)
{
    if (!ne)
    {
        return;
    }
    free(ne->primary_diagonal);
    free(ne->eliminated_diagonal);
    free(ne->primary_gradient);
    free(ne->eliminated_gradient);
    free(ne->cross_primary);
    free(ne->cross_eliminated);
    free(ne->cross_next);
    free(ne->cross_values);
    free(ne->adjacency_head);
    free(ne->adjacency_tail);
    free(ne->adjacency_size);
    free(ne->pc_row);
    free(ne->pc_col);
    free(ne->pc_values);
    free(ne);
}

/* findOrCreateCrossBlock, block_normal_equations.cpp:85-106 */
static int64_t FN(orc_ne_cross)(NE* ne, int64_t primary, int64_t eliminated)
{
    for (int64_t c = ne->adjacency_head[eliminated]; c >= 0; c = ne->cross_next[c])
    {
        if (ne->cross_primary[c] == primary)
        {
            return c;
        }
    }
    if (ne->cross_count == ne->cross_capacity)
    {
        const int64_t capacity = ne->cross_capacity ? ne->cross_capacity * 2 : 64;
        ne->cross_primary = (int64_t*)realloc(ne->cross_primary, (size_t)capacity * sizeof(int64_t));
        ne->cross_eliminated = (int64_t*)realloc(ne->cross_eliminated, (size_t)capacity * sizeof(int64_t));
        ne->cross_next = (int64_t*)realloc(ne->cross_next, (size_t)capacity * sizeof(int64_t));
        ne->cross_values =
            (S*)realloc(ne->cross_values, (size_t)(capacity * ne->bp * ne->bl) * sizeof(S));
        ne->cross_capacity = capacity;
    }
    const int64_t c = ne->cross_count++;
    ne->cross_primary[c] = primary;
    ne->cross_eliminated[c] = eliminated;
    ne->cross_next[c] = -1;
    memset(ne->cross_values + c * ne->bp * ne->bl, 0, (size_t)(ne->bp * ne->bl) * sizeof(S));
    if (ne->adjacency_tail[eliminated] < 0)
    {
        ne->adjacency_head[eliminated] = c;
    }
    else
    {
        ne->cross_next[ne->adjacency_tail[eliminated]] = c;
    }
    ne->adjacency_tail[eliminated] = c;
    ne->adjacency_size[eliminated] += 1;
    return c;
}

/* findOrCreatePrimaryCrossBlock, block_normal_equations.cpp:109-133 */
static int64_t FN(orc_ne_primary_cross)(NE* ne, int64_t row_block, int64_t column_block)
{
    for (int64_t index = 0; index < ne->pc_count; ++index)
    {
        if (ne->pc_row[index] == row_block && ne->pc_col[index] == column_block)
        {
            return index;
        }
    }
    if (ne->pc_count == ne->pc_capacity)
    {
        const int64_t capacity = ne->pc_capacity ? ne->pc_capacity * 2 : 16;
        ne->pc_row = (int64_t*)realloc(ne->pc_row, (size_t)capacity * sizeof(int64_t));
        ne->pc_col = (int64_t*)realloc(ne->pc_col, (size_t)capacity * sizeof(int64_t));
        ne->pc_values = (S*)realloc(ne->pc_values, (size_t)(capacity * ne->bp * ne->bp) * sizeof(S));
        ne->pc_capacity = capacity;
    }
    const int64_t index = ne->pc_count++;
    ne->pc_row[index] = row_block;
    ne->pc_col[index] = column_block;
    memset(ne->pc_values + index * ne->bp * ne->bp, 0, (size_t)(ne->bp * ne->bp) * sizeof(S));
    return index;
}

/* validateResidual, block_normal_equations.cpp:47-82 */
static int FN(orc_ne_validate)(const S* jacobian, int64_t jacobian_size, const S* residual,
                               int64_t residual_size, S weight, const char* operation)
{
    if (!jacobian || !residual || residual_size <= 0)
    {
        return orc_fail(ORC_INVALID_ARGUMENT, "%s: pointers must be non-null and residual size positive",
                        operation);
    }
    if (!isfinite(weight) || weight < (S)0)
    {
        return orc_fail(ORC_INVALID_ARGUMENT, "%s: weight must be finite and non-negative", operation);
    }
    for (int64_t index = 0; index < jacobian_size; ++index)
    {
        if (!isfinite(jacobian[index]))
        {
            return orc_fail(ORC_INVALID_ARGUMENT, "%s: Jacobian values must be finite", operation);
        }
    }
    for (int64_t index = 0; index < residual_size; ++index)
    {
        if (!isfinite(residual[index]))
        {
            return orc_fail(ORC_INVALID_ARGUMENT, "%s: residual values must be finite", operation);
        }
    }
    return ORC_OK;
}

/* addPrimaryTerms, block_normal_equations.cpp:136-222 */
static int FN(orc_ne_primary_terms)(NE* ne, int64_t count, const int64_t* blocks,
                                    const S* jacobians, const S* residual, int64_t m, S weight)
{
    const int64_t bp = ne->bp;
    if (count <= 0)
    {
        return orc_fail(ORC_INVALID_ARGUMENT,
                        "BlockNormalEquations: primary block and Jacobian lists must have equal non-zero size");
    }
    for (int64_t index = 0; index < count; ++index)
    {
        const int64_t block = blocks[index];
        if (block < 0 || block >= ne->P)
        {
            return orc_fail(ORC_OUT_OF_RANGE, "BlockNormalEquations: primary block index out of range");
        }
        for (int64_t before = 0; before < index; ++before)
        {
            if (blocks[before] == block)
            {
                return orc_fail(ORC_INVALID_ARGUMENT,
                                "BlockNormalEquations: primary block indices must be unique");
            }
        }
        const int status = FN(orc_ne_validate)(jacobians + index * m * bp, m * bp, residual, m, weight,
                                               "BlockNormalEquations::addPrimaryTerms");
        if (status != ORC_OK)
        {
            return status;
        }
    }
    for (int64_t block_index = 0; block_index < count; ++block_index)
    {
        const int64_t block = blocks[block_index];
        const S* jacobian = jacobians + block_index * m * bp;
        const int64_t matrix_offset = block * bp * bp;
        const int64_t gradient_offset = block * bp;
        for (int64_t row = 0; row < m; ++row)
        {
            for (int64_t column = 0; column < bp; ++column)
            {
                const S value = jacobian[row * bp + column];
                ne->primary_gradient[gradient_offset + column] += weight * value * residual[row];
                for (int64_t other = 0; other < bp; ++other)
                {
                    ne->primary_diagonal[matrix_offset + column * bp + other] +=
                        weight * value * jacobian[row * bp + other];
                }
            }
        }
    }
    for (int64_t left = 0; left < count; ++left)
    {
        for (int64_t right = left + 1; right < count; ++right)
        {
            const int ordered = blocks[left] < blocks[right];
            const int64_t row_block = ordered ? blocks[left] : blocks[right];
            const int64_t column_block = ordered ? blocks[right] : blocks[left];
            const S* row_jacobian = jacobians + (ordered ? left : right) * m * bp;
            const S* column_jacobian = jacobians + (ordered ? right : left) * m * bp;
            const int64_t cross_index = FN(orc_ne_primary_cross)(ne, row_block, column_block);
            S* cross = ne->pc_values + cross_index * bp * bp; /* after any realloc */
            for (int64_t residual_row = 0; residual_row < m; ++residual_row)
            {
                for (int64_t row = 0; row < bp; ++row)
                {
                    const S row_value = row_jacobian[residual_row * bp + row];
                    for (int64_t column = 0; column < bp; ++column)
                    {
                        cross[row * bp + column] +=
                            weight * row_value * column_jacobian[residual_row * bp + column];
                    }
                }
            }
        }
    }
    return ORC_OK;
}

static void FN(orc_ne_eliminated_terms)(NE* ne, int64_t eliminated, const S* jacobian,
                                        const S* residual, int64_t m, S weight)
{
    const int64_t bl = ne->bl;
    const int64_t matrix_offset = eliminated * bl * bl;
    const int64_t gradient_offset = eliminated * bl;
    for (int64_t row = 0; row < m; ++row)
    {
        for (int64_t col = 0; col < bl; ++col)
        {
            const S value = jacobian[row * bl + col];
            ne->eliminated_gradient[gradient_offset + col] += weight * value * residual[row];
            for (int64_t other = 0; other < bl; ++other)
            {
                ne->eliminated_diagonal[matrix_offset + col * bl + other] +=
                    weight * value * jacobian[row * bl + other];
            }
        }
    }
}

int FN(orc_ne_add_residual)(NE* ne, int64_t primary_count_in_residual, const int64_t* primaries,
                            const S* primary_jacobians, int64_t eliminated,
                            const S* eliminated_jacobian, const S* residual, int64_t m, S weight)
{
    const int64_t bp = ne->bp, bl = ne->bl;
    if (primary_count_in_residual <= 0)
    {
        /* addEliminatedResidualBlock, block_normal_equations.cpp:338-373 */
        if (eliminated < 0 || eliminated >= ne->L)
        {
            return orc_fail(ORC_OUT_OF_RANGE,
                            "BlockNormalEquations::addEliminatedResidualBlock: block index out of range");
        }
        const int status = FN(orc_ne_validate)(eliminated_jacobian, m * bl, residual, m, weight,
                                               "BlockNormalEquations::addEliminatedResidualBlock");
        if (status != ORC_OK)
        {
            return status;
        }
        FN(orc_ne_eliminated_terms)(ne, eliminated, eliminated_jacobian, residual, m, weight);
        return ORC_OK;
    }
    if (eliminated < 0)
    {
        /* addPrimaryResidualBlocks, block_normal_equations.cpp:326-335 */
        return FN(orc_ne_primary_terms)(ne, primary_count_in_residual, primaries, primary_jacobians,
                                        residual, m, weight);
    }
    /* addResidualBlocks, block_normal_equations.cpp:243-312 */
    if (eliminated >= ne->L)
    {
        return orc_fail(ORC_OUT_OF_RANGE,
                        "BlockNormalEquations::addResidualBlocks: eliminated block out of range");
    }
    int status = FN(orc_ne_validate)(eliminated_jacobian, m * bl, residual, m, weight,
                                     "BlockNormalEquations::addResidualBlocks(eliminated)");
    if (status != ORC_OK)
    {
        return status;
    }
    status = FN(orc_ne_primary_terms)(ne, primary_count_in_residual, primaries, primary_jacobians,
                                      residual, m, weight);
    if (status != ORC_OK)
    {
        return status;
    }
    for (int64_t primary_index = 0; primary_index < primary_count_in_residual; ++primary_index)
    {
        const int64_t cross_index = FN(orc_ne_cross)(ne, primaries[primary_index], eliminated);
        S* cross = ne->cross_values + cross_index * bp * bl; /* after any realloc */
        const S* primary_jacobian = primary_jacobians + primary_index * m * bp;
        for (int64_t row = 0; row < m; ++row)
        {
            for (int64_t primary_column = 0; primary_column < bp; ++primary_column)
            {
                const S primary_value = primary_jacobian[row * bp + primary_column];
                for (int64_t eliminated_column = 0; eliminated_column < bl; ++eliminated_column)
                {
                    cross[primary_column * bl + eliminated_column] +=
                        weight * primary_value * eliminated_jacobian[row * bl + eliminated_column];
                }
            }
        }
    }
    FN(orc_ne_eliminated_terms)(ne, eliminated, eliminated_jacobian, residual, m, weight);
    return ORC_OK;
}

int FN(orc_ne_add_observations)(NE* ne, int64_t count, int64_t m, const int64_t* primaries,
                                const int64_t* eliminated, const S* primary_jacobians,
                                const S* eliminated_jacobians, const S* residuals, S huber_delta)
{
    for (int64_t i = 0; i < count; ++i)
    {
        const S* r = residuals + i * m;
        S squared = (S)0;
        for (int64_t k = 0; k < m; ++k)
        {
            squared += r[k] * r[k];
        }
        S cost, weight;
        int status = FN(orc_huber)(squared, huber_delta, &cost, &weight);
        if (status == ORC_OK)
        {
            status = FN(orc_ne_add_residual)(ne, 1, primaries + i, primary_jacobians + i * m * ne->bp,
                                             eliminated[i], eliminated_jacobians + i * m * ne->bl, r, m,
                                             weight);
        }
        if (status != ORC_OK)
        {
            return status;
        }
    }
    return ORC_OK;
}

/* mergeFrom, block_normal_equations.cpp:376-411 */
int FN(orc_ne_merge)(NE* target, const NE* source)
{
    if (target->P != source->P || target->L != source->L || target->bp != source->bp ||
        target->bl != source->bl)
    {
        return orc_fail(ORC_INVALID_ARGUMENT, "BlockNormalEquations::mergeFrom: block layouts must match");
    }
    const int64_t bp = target->bp, bl = target->bl;
    for (int64_t i = 0; i < target->P * bp * bp; ++i)
    {
        target->primary_diagonal[i] += source->primary_diagonal[i];
    }
    for (int64_t i = 0; i < target->L * bl * bl; ++i)
    {
        target->eliminated_diagonal[i] += source->eliminated_diagonal[i];
    }
    for (int64_t i = 0; i < target->P * bp; ++i)
    {
        target->primary_gradient[i] += source->primary_gradient[i];
    }
    for (int64_t i = 0; i < target->L * bl; ++i)
    {
        target->eliminated_gradient[i] += source->eliminated_gradient[i];
    }
    for (int64_t k = 0; k < source->pc_count; ++k)
    {
        const int64_t index = FN(orc_ne_primary_cross)(target, source->pc_row[k], source->pc_col[k]);
        S* values = target->pc_values + index * bp * bp;
        for (int64_t i = 0; i < bp * bp; ++i)
        {
            values[i] += source->pc_values[k * bp * bp + i];
        }
    }
    for (int64_t c = 0; c < source->cross_count; ++c)
    {
        const int64_t index = FN(orc_ne_cross)(target, source->cross_primary[c], source->cross_eliminated[c]);
        S* values = target->cross_values + index * bp * bl;
        for (int64_t i = 0; i < bp * bl; ++i)
        {
            values[i] += source->cross_values[c * bp * bl + i];
        }
    }
    return ORC_OK;
}

void FN(orc_ne_counts)(const NE* ne, int64_t* cross_count, int64_t* primary_cross_count)
{
    *cross_count = ne->cross_count;
    *primary_cross_count = ne->pc_count;
}

void FN(orc_ne_export)(const NE* ne, S* primary_diagonal, S* eliminated_diagonal, S* primary_gradient,
                       S* eliminated_gradient, int64_t* adjacency_offsets, int64_t* cross_primary,
                       S* cross_values, int64_t* primary_cross_row, int64_t* primary_cross_col,
                       S* primary_cross_values)
{
    const int64_t bp = ne->bp, bl = ne->bl;
    if (primary_diagonal)
        memcpy(primary_diagonal, ne->primary_diagonal, (size_t)(ne->P * bp * bp) * sizeof(S));
    if (eliminated_diagonal)
        memcpy(eliminated_diagonal, ne->eliminated_diagonal, (size_t)(ne->L * bl * bl) * sizeof(S));
    if (primary_gradient)
        memcpy(primary_gradient, ne->primary_gradient, (size_t)(ne->P * bp) * sizeof(S));
    if (eliminated_gradient)
        memcpy(eliminated_gradient, ne->eliminated_gradient, (size_t)(ne->L * bl) * sizeof(S));
    int64_t k = 0;
    for (int64_t l = 0; l < ne->L; ++l)
    {
        if (adjacency_offsets)
            adjacency_offsets[l] = k;
        for (int64_t c = ne->adjacency_head[l]; c >= 0; c = ne->cross_next[c], ++k)
        {
            if (cross_primary)
                cross_primary[k] = ne->cross_primary[c];
            if (cross_values)
                memcpy(cross_values + k * bp * bl, ne->cross_values + c * bp * bl,
                       (size_t)(bp * bl) * sizeof(S));
        }
    }
    if (adjacency_offsets)
        adjacency_offsets[ne->L] = k;
    for (int64_t p = 0; p < ne->pc_count; ++p)
    {
        if (primary_cross_row)
            primary_cross_row[p] = ne->pc_row[p];
        if (primary_cross_col)
            primary_cross_col[p] = ne->pc_col[p];
        if (primary_cross_values)
            memcpy(primary_cross_values + p * bp * bp, ne->pc_values + p * bp * bp,
                   (size_t)(bp * bp) * sizeof(S));
    }
}

/* ===================================================================== small linear algebra
 * block_schur_linear_algebra.h. */
static int FN(orc_invert_spd)(const S* matrix, int64_t size, S* inverse, S* lower, S* intermediate)
{
    /* invertPositiveDefiniteInto, block_schur_linear_algebra.h:91-147 (same arithmetic as
     * invertPositiveDefinite :30-89) */
    for (int64_t i = 0; i < size * size; ++i)
    {
        lower[i] = (S)0;
    }
    for (int64_t row = 0; row < size; ++row)
    {
        for (int64_t column = 0; column <= row; ++column)
        {
            S value = matrix[row * size + column];
            for (int64_t inner = 0; inner < column; ++inner)
            {
                value -= lower[row * size + inner] * lower[column * size + inner];
            }
            if (row == column)
            {
                if (!(value > (S)0) || !isfinite(value))
                {
                    return 0;
                }
                lower[row * size + column] = (S)sqrt(value);
            }
            else
            {
                lower[row * size + column] = value / lower[column * size + column];
            }
        }
    }
    for (int64_t i = 0; i < size * size; ++i)
    {
        inverse[i] = (S)0;
    }
    for (int64_t column = 0; column < size; ++column)
    {
        for (int64_t row = 0; row < size; ++row)
        {
            S value = row == column ? (S)1 : (S)0;
            for (int64_t inner = 0; inner < row; ++inner)
            {
                value -= lower[row * size + inner] * intermediate[inner];
            }
            intermediate[row] = value / lower[row * size + row];
        }
        for (int64_t offset = 0; offset < size; ++offset)
        {
            const int64_t row = size - 1 - offset;
            S value = intermediate[row];
            for (int64_t inner = row + 1; inner < size; ++inner)
            {
                value -= lower[inner * size + row] * inverse[inner * size + column];
            }
            inverse[row * size + column] = value / lower[row * size + row];
        }
    }
    return 1;
}

/* multiplyMatrixVector :181-196 */
static void FN(orc_mat_vec)(const S* matrix, int64_t rows, int64_t cols, const S* vector, S* result)
{
    for (int64_t row = 0; row < rows; ++row)
    {
        S value = (S)0;
        for (int64_t col = 0; col < cols; ++col)
        {
            value += matrix[row * cols + col] * vector[col];
        }
        result[row] = value;
    }
}

/* addMatrixVector :198-215 */
static void FN(orc_add_mat_vec)(const S* matrix, int64_t rows, int64_t cols, const S* vector, S scale,
                                S* result)
{
    for (int64_t row = 0; row < rows; ++row)
    {
        S value = (S)0;
        for (int64_t col = 0; col < cols; ++col)
        {
            value += matrix[row * cols + col] * vector[col];
        }
        result[row] += scale * value;
    }
}

/* addTransposeMatrixVector :217-233 */
static void FN(orc_add_mat_t_vec)(const S* matrix, int64_t rows, int64_t cols, const S* vector, S* result)
{
    for (int64_t col = 0; col < cols; ++col)
    {
        S value = (S)0;
        for (int64_t row = 0; row < rows; ++row)
        {
            value += matrix[row * cols + col] * vector[row];
        }
        result[col] += value;
    }
}

static S FN(orc_dot)(int64_t n, const S* a, const S* b)
{
    S result = (S)0;
    for (int64_t i = 0; i < n; ++i)
    {
        result += a[i] * b[i];
    }
    return result;
}

static S FN(orc_norm)(int64_t n, const S* a)
{
    const S d = FN(orc_dot)(n, a, a);
    return (S)sqrt(d > (S)0 ? d : (S)0);
}

/* transformed cross row `row` = Hll^-1 * W[row] (block_schur.cpp:205-217, transform9x3 and the
 * generic multiplyMatrixVector loop evaluate the same sums in the same order). */
static void FN(orc_transform_cross)(const S* inverse, const S* cross, int64_t bp, int64_t bl, S* transformed)
{
    for (int64_t row = 0; row < bp; ++row)
    {
        FN(orc_mat_vec)(inverse, bl, bl, cross + row * bl, transformed + row * bl);
    }
}

/* ===================================================================== Schur pattern
 * block_schur_sparse_assembly.h:41-260 (rebuild).  The slot set is ordered by
 * (row, col) exactly like the reference's std::map; this restatement builds it
 * by sorting instead of the reference's O(rows x slots) expansion loop. */
typedef struct
{
    int64_t block_count;
    int64_t* block_row; /* slot -> block row */
    int64_t* block_col; /* slot -> block column */
    int64_t* block_row_start; /* P+1: first slot of each block row */
} FN(orc_pattern);

static int FN(orc_pattern_build)(const NE* ne, FN(orc_pattern)* pattern)
{
    int64_t pairs = ne->P + 2 * ne->pc_count;
    for (int64_t l = 0; l < ne->L; ++l)
    {
        pairs += ne->adjacency_size[l] * ne->adjacency_size[l];
    }
    int64_t* rows = (int64_t*)malloc((size_t)(pairs + 1) * sizeof(int64_t));
    int64_t* cols = (int64_t*)malloc((size_t)(pairs + 1) * sizeof(int64_t));
    int64_t* order = (int64_t*)malloc((size_t)(pairs + 1) * sizeof(int64_t));
    if (!rows || !cols || !order)
    {
        free(rows);
        free(cols);
        free(order);
        return orc_fail(ORC_NO_MEMORY, "oracle: out of memory");
    }
    int64_t k = 0;
    for (int64_t p = 0; p < ne->P; ++p)
    {
        rows[k] = p;
        cols[k++] = p;
    }
    for (int64_t c = 0; c < ne->pc_count; ++c)
    {
        rows[k] = ne->pc_row[c];
        cols[k++] = ne->pc_col[c];
        rows[k] = ne->pc_col[c];
        cols[k++] = ne->pc_row[c];
    }
    for (int64_t l = 0; l < ne->L; ++l)
    {
        for (int64_t a = ne->adjacency_head[l]; a >= 0; a = ne->cross_next[a])
        {
            for (int64_t b = ne->adjacency_head[l]; b >= 0; b = ne->cross_next[b])
            {
                rows[k] = ne->cross_primary[a];
                cols[k++] = ne->cross_primary[b];
            }
        }
    }
    int status = orc_stable_sort_pairs(pairs, rows, cols, order);
    if (status != ORC_OK)
    {
        free(rows);
        free(cols);
        free(order);
        return status;
    }
    pattern->block_row = (int64_t*)malloc((size_t)(pairs + 1) * sizeof(int64_t));
    pattern->block_col = (int64_t*)malloc((size_t)(pairs + 1) * sizeof(int64_t));
    pattern->block_row_start = (int64_t*)calloc((size_t)ne->P + 2, sizeof(int64_t));
    int64_t count = 0;
    for (int64_t i = 0; i < pairs; ++i)
    {
        const int64_t r = rows[order[i]], c = cols[order[i]];
        if (count > 0 && pattern->block_row[count - 1] == r && pattern->block_col[count - 1] == c)
        {
            continue;
        }
        pattern->block_row[count] = r;
        pattern->block_col[count] = c;
        pattern->block_row_start[r + 1] += 1;
        ++count;
    }
    for (int64_t p = 0; p < ne->P; ++p)
    {
        pattern->block_row_start[p + 1] += pattern->block_row_start[p];
    }
    pattern->block_count = count;
    free(rows);
    free(cols);
    free(order);
    return ORC_OK;
}

static void FN(orc_pattern_free)(FN(orc_pattern)* pattern)
{
    free(pattern->block_row);
    free(pattern->block_col);
    free(pattern->block_row_start);
}

/* slot index of (row, col): binary search inside the block row */
static int64_t FN(orc_pattern_slot)(const FN(orc_pattern)* pattern, int64_t row, int64_t col)
{
    int64_t lo = pattern->block_row_start[row], hi = pattern->block_row_start[row + 1];
    while (lo < hi)
    {
        const int64_t mid = (lo + hi) / 2;
        if (pattern->block_col[mid] < col)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

/* valuePosition, block_schur_sparse_assembly.h:262-272: each block row owns
 * bp scalar rows of (slots in the row) * bp entries; columns ascend. */
static int64_t FN(orc_value_position)(const FN(orc_pattern)* pattern, int64_t bp, int64_t slot,
                                      int64_t local_row, int64_t local_col)
{
    const int64_t block_row = pattern->block_row[slot];
    const int64_t row_start = pattern->block_row_start[block_row];
    const int64_t row_slots = pattern->block_row_start[block_row + 1] - row_start;
    return row_start * bp * bp + local_row * row_slots * bp + (slot - row_start) * bp + local_col;
}

int FN(orc_schur_pattern_nnz)(const NE* ne, int64_t* nnz, int64_t* block_count)
{
    FN(orc_pattern) pattern;
    const int status = FN(orc_pattern_build)(ne, &pattern);
    if (status != ORC_OK)
        return status;
    *block_count = pattern.block_count;
    *nnz = pattern.block_count * ne->bp * ne->bp;
    FN(orc_pattern_free)(&pattern);
    return ORC_OK;
}

/* Damping (block_schur.cpp:106-120) and eliminated inverses (:122-149). */
static int FN(orc_damped_blocks)(const NE* ne, S damping, S minimum_diagonal, S* primary_diagonal,
                                 S* eliminated_diagonal, S* eliminated_inverse)
{
    const int64_t bp = ne->bp, bl = ne->bl;
    memcpy(primary_diagonal, ne->primary_diagonal, (size_t)(ne->P * bp * bp) * sizeof(S));
    memcpy(eliminated_diagonal, ne->eliminated_diagonal, (size_t)(ne->L * bl * bl) * sizeof(S));
    for (int64_t block = 0; block < ne->P; ++block)
    {
        for (int64_t d = 0; d < bp; ++d)
        {
            S* value = primary_diagonal + block * bp * bp + d * bp + d;
            const S magnitude = (S)fabs((double)*value);
            *value += damping * (magnitude > minimum_diagonal ? magnitude : minimum_diagonal);
        }
    }
    for (int64_t block = 0; block < ne->L; ++block)
    {
        for (int64_t d = 0; d < bl; ++d)
        {
            S* value = eliminated_diagonal + block * bl * bl + d * bl + d;
            const S magnitude = (S)fabs((double)*value);
            *value += damping * (magnitude > minimum_diagonal ? magnitude : minimum_diagonal);
        }
    }
    S* lower = (S*)malloc((size_t)(bl * bl + bl) * sizeof(S));
    for (int64_t block = 0; block < ne->L; ++block)
    {
        if (!FN(orc_invert_spd)(eliminated_diagonal + block * bl * bl, bl,
                                eliminated_inverse + block * bl * bl, lower, lower + bl * bl))
        {
            free(lower);
            return 0;
        }
    }
    free(lower);
    return 1;
}

/* Reduced RHS, block_schur.cpp:151-177. */
static void FN(orc_reduced_rhs)(const NE* ne, const S* eliminated_inverse, S* rhs)
{
    const int64_t bp = ne->bp, bl = ne->bl;
    for (int64_t i = 0; i < ne->P * bp; ++i)
    {
        rhs[i] = -ne->primary_gradient[i];
    }
    S* product = (S*)malloc((size_t)bl * sizeof(S));
    for (int64_t l = 0; l < ne->L; ++l)
    {
        FN(orc_mat_vec)(eliminated_inverse + l * bl * bl, bl, bl, ne->eliminated_gradient + l * bl, product);
        for (int64_t c = ne->adjacency_head[l]; c >= 0; c = ne->cross_next[c])
        {
            FN(orc_add_mat_vec)(ne->cross_values + c * bp * bl, bp, bl, product, (S)1,
                                rhs + ne->cross_primary[c] * bp);
        }
    }
    free(product);
}

/* Block-Jacobi preconditioner blocks, block_schur.cpp:179-250.  Crosses of a
 * primary are visited in creation order (the reference's primary_adjacency). */
static int FN(orc_preconditioner)(const NE* ne, const S* primary_diagonal, const S* eliminated_inverse,
                                  S* inverse_blocks)
{
    const int64_t bp = ne->bp, bl = ne->bl;
    int64_t* first = (int64_t*)malloc(((size_t)ne->P + 1) * sizeof(int64_t));
    int64_t* next = (int64_t*)malloc(((size_t)ne->cross_count + 1) * sizeof(int64_t));
    int64_t* last = (int64_t*)malloc(((size_t)ne->P + 1) * sizeof(int64_t));
    for (int64_t p = 0; p < ne->P; ++p)
    {
        first[p] = -1;
        last[p] = -1;
    }
    for (int64_t c = 0; c < ne->cross_count; ++c)
    {
        const int64_t p = ne->cross_primary[c];
        next[c] = -1;
        if (last[p] < 0)
            first[p] = c;
        else
            next[last[p]] = c;
        last[p] = c;
    }
    S* schur = (S*)malloc((size_t)(bp * bp) * sizeof(S));
    S* temporary = (S*)malloc((size_t)(bp * bl) * sizeof(S));
    S* lower = (S*)malloc((size_t)(bp * bp + bp) * sizeof(S));
    int ok = 1;
    for (int64_t block = 0; block < ne->P && ok; ++block)
    {
        memcpy(schur, primary_diagonal + block * bp * bp, (size_t)(bp * bp) * sizeof(S));
        for (int64_t c = first[block]; c >= 0; c = next[c])
        {
            const S* cross = ne->cross_values + c * bp * bl;
            FN(orc_transform_cross)(eliminated_inverse + ne->cross_eliminated[c] * bl * bl, cross, bp, bl,
                                    temporary);
            for (int64_t row = 0; row < bp; ++row)
            {
                for (int64_t col = 0; col < bp; ++col)
                {
                    const S* transformed = temporary + row * bl;
                    const S* source_row = cross + col * bl;
                    S value = (S)0;
                    if (bl == 3)
                    {
                        value = transformed[0] * source_row[0] + transformed[1] * source_row[1] +
                                transformed[2] * source_row[2];
                    }
                    else
                    {
                        for (int64_t inner = 0; inner < bl; ++inner)
                            value += transformed[inner] * source_row[inner];
                    }
                    schur[row * bp + col] -= value;
                }
            }
        }
        ok = FN(orc_invert_spd)(schur, bp, inverse_blocks + block * bp * bp, lower, lower + bp * bp);
    }
    free(first);
    free(next);
    free(last);
    free(schur);
    free(temporary);
    free(lower);
    return ok;
}

/* Scalar CSR values of the reduced Schur complement: CPU branch of
 * assembleReducedSchurCsr, block_schur_sparse_assembly.h:812-910. */
static void FN(orc_assemble_csr)(const NE* ne, const FN(orc_pattern)* pattern, const S* primary_diagonal,
                                 const S* eliminated_inverse, S* values)
{
    const int64_t bp = ne->bp, bl = ne->bl;
    memset(values, 0, (size_t)(pattern->block_count * bp * bp) * sizeof(S));
    for (int64_t block = 0; block < ne->P; ++block)
    {
        const int64_t slot = FN(orc_pattern_slot)(pattern, block, block);
        for (int64_t row = 0; row < bp; ++row)
            for (int64_t column = 0; column < bp; ++column)
                values[FN(orc_value_position)(pattern, bp, slot, row, column)] +=
                    primary_diagonal[block * bp * bp + row * bp + column];
    }
    for (int64_t index = 0; index < ne->pc_count; ++index)
    {
        const int64_t forward = FN(orc_pattern_slot)(pattern, ne->pc_row[index], ne->pc_col[index]);
        const int64_t transpose = FN(orc_pattern_slot)(pattern, ne->pc_col[index], ne->pc_row[index]);
        const S* cross = ne->pc_values + index * bp * bp;
        for (int64_t row = 0; row < bp; ++row)
        {
            for (int64_t column = 0; column < bp; ++column)
            {
                values[FN(orc_value_position)(pattern, bp, forward, row, column)] += cross[row * bp + column];
                values[FN(orc_value_position)(pattern, bp, transpose, column, row)] += cross[row * bp + column];
            }
        }
    }
    int64_t max_adjacency = 1;
    for (int64_t l = 0; l < ne->L; ++l)
        if (ne->adjacency_size[l] > max_adjacency)
            max_adjacency = ne->adjacency_size[l];
    S* transformed = (S*)malloc((size_t)(max_adjacency * bp * bl) * sizeof(S));
    int64_t* entries = (int64_t*)malloc((size_t)max_adjacency * sizeof(int64_t));
    for (int64_t l = 0; l < ne->L; ++l)
    {
        int64_t k = 0;
        for (int64_t c = ne->adjacency_head[l]; c >= 0; c = ne->cross_next[c])
        {
            entries[k] = c;
            FN(orc_transform_cross)(eliminated_inverse + l * bl * bl, ne->cross_values + c * bp * bl, bp, bl,
                                    transformed + k * bp * bl);
            ++k;
        }
        for (int64_t left = 0; left < k; ++left)
        {
            for (int64_t right = 0; right < k; ++right)
            {
                const S* right_cross = ne->cross_values + entries[right] * bp * bl;
                const int64_t slot = FN(orc_pattern_slot)(pattern, ne->cross_primary[entries[left]],
                                                          ne->cross_primary[entries[right]]);
                for (int64_t row = 0; row < bp; ++row)
                {
                    for (int64_t column = 0; column < bp; ++column)
                    {
                        S value = (S)0;
                        for (int64_t inner = 0; inner < bl; ++inner)
                        {
                            value += transformed[left * bp * bl + row * bl + inner] *
                                     right_cross[column * bl + inner];
                        }
                        values[FN(orc_value_position)(pattern, bp, slot, row, column)] += -value;
                    }
                }
            }
        }
    }
    free(transformed);
    free(entries);
}

int FN(orc_schur_system)(const NE* ne, S damping, S minimum_diagonal, int64_t* row_offsets,
                         int64_t* col_indices, S* values, S* rhs, S* preconditioner_inverse)
{
    const int64_t bp = ne->bp, bl = ne->bl;
    S* primary_diagonal = (S*)malloc((size_t)(ne->P * bp * bp + 1) * sizeof(S));
    S* eliminated_diagonal = (S*)malloc((size_t)(ne->L * bl * bl + 1) * sizeof(S));
    S* eliminated_inverse = (S*)malloc((size_t)(ne->L * bl * bl + 1) * sizeof(S));
    int status = ORC_OK;
    FN(orc_pattern) pattern = {0, NULL, NULL, NULL};
    if (!FN(orc_damped_blocks)(ne, damping, minimum_diagonal, primary_diagonal, eliminated_diagonal,
                               eliminated_inverse))
    {
        status = orc_fail(ORC_RUNTIME_ERROR, "eliminated block is not positive definite");
        goto done;
    }
    status = FN(orc_pattern_build)(ne, &pattern);
    if (status != ORC_OK)
        goto done;
    if (row_offsets || col_indices)
    {
        int64_t cursor = 0;
        for (int64_t block_row = 0; block_row < ne->P; ++block_row)
        {
            for (int64_t local_row = 0; local_row < bp; ++local_row)
            {
                if (row_offsets)
                    row_offsets[block_row * bp + local_row] = cursor;
                for (int64_t slot = pattern.block_row_start[block_row];
                     slot < pattern.block_row_start[block_row + 1]; ++slot)
                {
                    for (int64_t column = 0; column < bp; ++column)
                    {
                        if (col_indices)
                            col_indices[cursor] = pattern.block_col[slot] * bp + column;
                        ++cursor;
                    }
                }
            }
        }
        if (row_offsets)
            row_offsets[ne->P * bp] = cursor;
    }
    if (values)
        FN(orc_assemble_csr)(ne, &pattern, primary_diagonal, eliminated_inverse, values);
    if (rhs)
        FN(orc_reduced_rhs)(ne, eliminated_inverse, rhs);
    if (preconditioner_inverse &&
        !FN(orc_preconditioner)(ne, primary_diagonal, eliminated_inverse, preconditioner_inverse))
    {
        status = orc_fail(ORC_RUNTIME_ERROR, "Schur preconditioner block is not positive definite");
    }
done:
    FN(orc_pattern_free)(&pattern);
    free(primary_diagonal);
    free(eliminated_diagonal);
    free(eliminated_inverse);
    return status;
}

/* ===================================================================== Schur solve
 * solveDampedSchurComplement, block_schur.cpp:54-459 with the CPU reduced PCG
 * (block_schur_cpu_solver.h:14-82) and the dense Cholesky backend
 * (block_schur_dense_solver.h:319-399; serial factor order). */
typedef struct
{
    const NE* ne;
    const S* primary_diagonal;
    const S* eliminated_inverse;
    const S* preconditioner;
    S* point;
    S* inverse_value;
} FN(orc_schur_ops);

/* apply_schur, block_schur.cpp:254-309 */
static void FN(orc_apply_schur)(const FN(orc_schur_ops)* ops, const S* input, S* output)
{
    const NE* ne = ops->ne;
    const int64_t bp = ne->bp, bl = ne->bl;
    for (int64_t i = 0; i < ne->P * bp; ++i)
        output[i] = (S)0;
    for (int64_t block = 0; block < ne->P; ++block)
        FN(orc_mat_vec)(ops->primary_diagonal + block * bp * bp, bp, bp, input + block * bp, output + block * bp);
    for (int64_t k = 0; k < ne->pc_count; ++k)
    {
        const S* values = ne->pc_values + k * bp * bp;
        FN(orc_add_mat_vec)(values, bp, bp, input + ne->pc_col[k] * bp, (S)1, output + ne->pc_row[k] * bp);
        FN(orc_add_mat_t_vec)(values, bp, bp, input + ne->pc_row[k] * bp, output + ne->pc_col[k] * bp);
    }
    for (int64_t l = 0; l < ne->L; ++l)
    {
        for (int64_t i = 0; i < bl; ++i)
            ops->point[i] = (S)0;
        for (int64_t c = ne->adjacency_head[l]; c >= 0; c = ne->cross_next[c])
            FN(orc_add_mat_t_vec)(ne->cross_values + c * bp * bl, bp, bl, input + ne->cross_primary[c] * bp,
                                  ops->point);
        FN(orc_mat_vec)(ops->eliminated_inverse + l * bl * bl, bl, bl, ops->point, ops->inverse_value);
        for (int64_t c = ne->adjacency_head[l]; c >= 0; c = ne->cross_next[c])
            FN(orc_add_mat_vec)(ne->cross_values + c * bp * bl, bp, bl, ops->inverse_value, (S)-1,
                                output + ne->cross_primary[c] * bp);
    }
}

static void FN(orc_apply_preconditioner)(const FN(orc_schur_ops)* ops, const S* input, S* output)
{
    const int64_t bp = ops->ne->bp;
    for (int64_t block = 0; block < ops->ne->P; ++block)
        FN(orc_mat_vec)(ops->preconditioner + block * bp * bp, bp, bp, input + block * bp, output + block * bp);
}

int FN(orc_schur_solve)(const NE* ne, S damping, const orc_schur_options* options, S* primary_step,
                        S* eliminated_step, orc_schur_report* report)
{
    memset(report, 0, sizeof(*report));
    if (!primary_step || !eliminated_step || (void*)primary_step == (void*)eliminated_step)
    {
        return orc_fail(ORC_INVALID_ARGUMENT,
                        "solveDampedSchurComplement: output vectors must be non-null and distinct");
    }
    if (!isfinite(damping) || damping < (S)0 || options->max_iterations <= 0 ||
        !isfinite(options->relative_tolerance) || options->relative_tolerance < 0 ||
        !isfinite(options->absolute_tolerance) || options->absolute_tolerance < 0 ||
        !isfinite(options->minimum_diagonal) || options->minimum_diagonal <= 0)
    {
        return orc_fail(ORC_INVALID_ARGUMENT, "solveDampedSchurComplement: invalid solver options");
    }
    const int64_t bp = ne->bp, bl = ne->bl;
    const int64_t n = ne->P * bp;
    const S rel = (S)options->relative_tolerance, abs_tol = (S)options->absolute_tolerance;
    if (!options->use_initial_guess)
        for (int64_t i = 0; i < n; ++i)
            primary_step[i] = (S)0;
    for (int64_t i = 0; i < ne->L * bl; ++i)
        eliminated_step[i] = (S)0;

    S* primary_diagonal = (S*)malloc((size_t)(ne->P * bp * bp + 1) * sizeof(S));
    S* eliminated_diagonal = (S*)malloc((size_t)(ne->L * bl * bl + 1) * sizeof(S));
    S* eliminated_inverse = (S*)malloc((size_t)(ne->L * bl * bl + 1) * sizeof(S));
    S* rhs = (S*)malloc((size_t)(n + 1) * sizeof(S));
    S* preconditioner = (S*)malloc((size_t)(ne->P * bp * bp + 1) * sizeof(S));
    S* work = (S*)malloc((size_t)(5 * n + 2 * bl + 8) * sizeof(S));
    FN(orc_pattern) pattern = {0, NULL, NULL, NULL};
    S* dense = NULL;
    S* point_rhs = NULL;
    int status = ORC_OK;

    if (!FN(orc_damped_blocks)(ne, damping, (S)options->minimum_diagonal, primary_diagonal,
                               eliminated_diagonal, eliminated_inverse))
    {
        snprintf(report->message, sizeof(report->message), "eliminated block is not positive definite");
        goto done;
    }
    FN(orc_reduced_rhs)(ne, eliminated_inverse, rhs);
    if (options->backend != ORC_BACKEND_DENSE_CPU &&
        !FN(orc_preconditioner)(ne, primary_diagonal, eliminated_inverse, preconditioner))
    {
        snprintf(report->message, sizeof(report->message), "Schur preconditioner block is not positive definite");
        goto done;
    }
    if (n == 0)
    {
        report->converged = 1;
    }
    else if (options->backend == ORC_BACKEND_DENSE_CPU)
    {
        /* assembleReducedSchurDenseLower + solveReducedSchurDenseLower */
        status = FN(orc_pattern_build)(ne, &pattern);
        if (status != ORC_OK)
            goto done;
        dense = (S*)malloc((size_t)(n * n) * sizeof(S));
        S* csr_values = (S*)malloc((size_t)(pattern.block_count * bp * bp) * sizeof(S));
        FN(orc_assemble_csr)(ne, &pattern, primary_diagonal, eliminated_inverse, csr_values);
        for (int64_t i = 0; i < n * n; ++i)
            dense[i] = (S)0;
        for (int64_t slot = 0; slot < pattern.block_count; ++slot)
            for (int64_t r = 0; r < bp; ++r)
                for (int64_t c = 0; c < bp; ++c)
                    dense[(pattern.block_row[slot] * bp + r) * n + pattern.block_col[slot] * bp + c] =
                        csr_values[FN(orc_value_position)(&pattern, bp, slot, r, c)];
        free(csr_values);
        for (int64_t i = 0; i < n; ++i)
            primary_step[i] = rhs[i];
        report->initial_residual_norm = (double)FN(orc_norm)(n, rhs);
        S* factor = (S*)malloc((size_t)(n * n) * sizeof(S));
        memcpy(factor, dense, (size_t)(n * n) * sizeof(S));
        int factored = 1;
        for (int64_t row = 0; row < n && factored; ++row)
        {
            for (int64_t column = 0; column <= row; ++column)
            {
                S dot = (S)0;
                for (int64_t inner = 0; inner < column; ++inner)
                    dot += factor[row * n + inner] * factor[column * n + inner];
                const S value = factor[row * n + column] - dot;
                if (row == column)
                {
                    if (!(value > (S)0) || !isfinite(value))
                    {
                        factored = 0;
                        break;
                    }
                    factor[row * n + column] = (S)sqrt(value);
                }
                else
                {
                    factor[row * n + column] = value / factor[column * n + column];
                }
            }
        }
        if (!factored)
        {
            snprintf(report->message, sizeof(report->message), "reduced Schur complement is not positive definite");
            free(factor);
        }
        else
        {
            for (int64_t row = 0; row < n; ++row)
            {
                S value = primary_step[row];
                for (int64_t inner = 0; inner < row; ++inner)
                    value -= factor[row * n + inner] * primary_step[inner];
                primary_step[row] = value / factor[row * n + row];
            }
            for (int64_t offset = 0; offset < n; ++offset)
            {
                const int64_t row = n - 1 - offset;
                S value = primary_step[row];
                for (int64_t inner = row + 1; inner < n; ++inner)
                    value -= factor[inner * n + row] * primary_step[inner];
                primary_step[row] = value / factor[row * n + row];
            }
            free(factor);
            S* residual = work;
            for (int64_t row = 0; row < n; ++row)
            {
                S product = (S)0;
                for (int64_t column = 0; column < n; ++column)
                    product += dense[row * n + column] * primary_step[column];
                residual[row] = rhs[row] - product;
            }
            report->final_residual_norm = (double)FN(orc_norm)(n, residual);
            const S tolerance = abs_tol + rel * (S)report->initial_residual_norm;
            const S floor_tol = (S)100 * (S)ORC_EPSILON *
                                ((S)report->initial_residual_norm > (S)1 ? (S)report->initial_residual_norm : (S)1);
            report->converged = isfinite(report->final_residual_norm) &&
                                (S)report->final_residual_norm <= (tolerance > floor_tol ? tolerance : floor_tol);
            report->iterations = 1;
            if (!report->converged)
                snprintf(report->message, sizeof(report->message), "dense Cholesky residual exceeds tolerance");
        }
    }
    else
    {
        /* solveReducedSchurOnCpu, block_schur_cpu_solver.h:14-82 */
        FN(orc_schur_ops) ops = {ne, primary_diagonal, eliminated_inverse, preconditioner,
                                 work + 5 * n, work + 5 * n + bl};
        S* product = work;
        S* residual = work + n;
        S* preconditioned = work + 2 * n;
        S* direction = work + 3 * n;
        FN(orc_apply_schur)(&ops, primary_step, product);
        for (int64_t i = 0; i < n; ++i)
            residual[i] = rhs[i] - product[i];
        S initial = FN(orc_norm)(n, residual);
        report->initial_residual_norm = (double)initial;
        report->final_residual_norm = (double)initial;
        const S tolerance = abs_tol + rel * initial;
        if (initial <= tolerance)
        {
            report->converged = 1;
        }
        else
        {
            FN(orc_apply_preconditioner)(&ops, residual, preconditioned);
            memcpy(direction, preconditioned, (size_t)n * sizeof(S));
            for (int64_t i = 0; i < n; ++i)
                product[i] = (S)0;
            S residual_dot = FN(orc_dot)(n, residual, preconditioned);
            for (int iteration = 0; iteration < options->max_iterations; ++iteration)
            {
                FN(orc_apply_schur)(&ops, direction, product);
                const S denominator = FN(orc_dot)(n, direction, product);
                if (!(denominator > (S)0) || !isfinite(denominator))
                {
                    snprintf(report->message, sizeof(report->message),
                             "reduced Schur complement is not positive definite");
                    break;
                }
                const S alpha = residual_dot / denominator;
                for (int64_t i = 0; i < n; ++i)
                {
                    primary_step[i] += alpha * direction[i];
                    residual[i] -= alpha * product[i];
                }
                report->iterations = iteration + 1;
                const S norm = FN(orc_norm)(n, residual);
                report->final_residual_norm = (double)norm;
                if (norm <= tolerance)
                {
                    report->converged = 1;
                    break;
                }
                FN(orc_apply_preconditioner)(&ops, residual, preconditioned);
                const S next_residual_dot = FN(orc_dot)(n, residual, preconditioned);
                const S beta = next_residual_dot / residual_dot;
                for (int64_t i = 0; i < n; ++i)
                    direction[i] = preconditioned[i] + beta * direction[i];
                residual_dot = next_residual_dot;
            }
        }
    }
    if (!report->converged)
    {
        if (report->message[0] == '\0')
            snprintf(report->message, sizeof(report->message), "PCG iteration limit reached");
        goto done;
    }
    /* back-substitution, block_schur.cpp:422-454 */
    point_rhs = (S*)malloc((size_t)bl * sizeof(S));
    for (int64_t l = 0; l < ne->L; ++l)
    {
        for (int64_t i = 0; i < bl; ++i)
            point_rhs[i] = -ne->eliminated_gradient[l * bl + i];
        for (int64_t c = ne->adjacency_head[l]; c >= 0; c = ne->cross_next[c])
        {
            const S* primary = primary_step + ne->cross_primary[c] * bp;
            const S* cross = ne->cross_values + c * bp * bl;
            for (int64_t column = 0; column < bl; ++column)
            {
                S value = (S)0;
                for (int64_t row = 0; row < bp; ++row)
                    value += cross[row * bl + column] * primary[row];
                point_rhs[column] -= value;
            }
        }
        FN(orc_mat_vec)(eliminated_inverse + l * bl * bl, bl, bl, point_rhs, eliminated_step + l * bl);
    }
    snprintf(report->message, sizeof(report->message), "converged");
done:
    FN(orc_pattern_free)(&pattern);
    free(dense);
    free(point_rhs);
    free(primary_diagonal);
    free(eliminated_diagonal);
    free(eliminated_inverse);
    free(rhs);
    free(preconditioner);
    free(work);
    return status;
}

#undef NE
#undef S
#undef FN
#undef ORC_CAT
#undef ORC_CAT2
