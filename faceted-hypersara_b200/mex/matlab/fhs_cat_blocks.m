function v = fhs_cat_blocks(y)
% FHS_CAT_BLOCKS  The reference's cell of cells y{l}{b} -> one column,
% channel after channel, blocks in order (the C ABI's layout).
parts = cell(numel(y), 1);
for l = 1:numel(y)
    parts{l} = vertcat(y{l}{:});
end
v = vertcat(parts{:});
end
