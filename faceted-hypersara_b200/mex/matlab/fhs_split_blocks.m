function y = fhs_split_blocks(v, blocks)
% FHS_SPLIT_BLOCKS  All channels' visibilities (one column, channel after
% channel, blocks in order) -> the reference's cell of cells y{l}{b}.
y = cell(numel(blocks), 1);
pos = 0;
for l = 1:numel(blocks)
    y{l} = cell(numel(blocks{l}), 1);
    for b = 1:numel(blocks{l})
        m = blocks{l}(b);
        y{l}{b} = v(pos + 1:pos + m);
        pos = pos + m;
    end
end
end
